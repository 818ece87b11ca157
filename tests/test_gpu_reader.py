"""GPU parity of the reader against the golden vectors of the reference and the CPU oracle.

Everything here calls the native library (``include/cubam_b200.h``) through
``cubam_b200``; the expected values come from ``tests/golden/`` (made by the
reference's own writer and reader code) and from ``oracle/bam_oracle.py``.
"""

import random
import struct
import zlib

import numpy as np
import pytest

from golden_io import GOLDEN, TAGS, bam_cases, batches, meta

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

import cubam_b200  # noqa: E402
from cubam_b200 import bgzf as G  # noqa: E402
from oracle import bam_oracle as O  # noqa: E402


def _np(t):
    return t.cpu().numpy()


def member(data: bytes, level: int = 6, strategy: int = zlib.Z_DEFAULT_STRATEGY, mem_level: int = 8) -> bytes:
    if not data:  # the reference accepts an empty member only in the exact form of the EOF member
        return G.EOF_BLOCK
    c = zlib.compressobj(level, zlib.DEFLATED, -15, mem_level, strategy)
    payload = c.compress(data) + c.flush()
    if len(payload) + 26 > 65536:  # does not shrink enough: a stored member, as BGZF writers do
        c = zlib.compressobj(0, zlib.DEFLATED, -15)
        payload = c.compress(data) + c.flush()
    bsize = 18 + len(payload) + 8
    if bsize > 65536:
        raise OverflowError("does not fit a BGZF member")
    head = b"\x1f\x8b\x08\x04\x00\x00\x00\x00\x00\xff\x06\x00BC\x02\x00" + struct.pack("<H", bsize - 1)
    return head + payload + struct.pack("<II", zlib.crc32(data) & 0xFFFFFFFF, len(data))


@pytest.mark.parametrize(("name", "chunk"), bam_cases())
def test_read_bam_matches_reference(tmp_path, name, chunk):
    path = GOLDEN / name
    got = list(cubam_b200.read_bam(path, chunk_bytes=chunk, piece=chunk // 2 + 1))
    exp = batches(name, chunk)
    assert len(got) == len(exp)
    for b, e in zip(got, exp):
        assert int(b.data.numel()) == e["data_size"]
        assert _np(b.offset).tolist() == e["offset"].tolist()
        for k in cubam_b200.RecordBatch.FIELDS:
            col = _np(getattr(b, k))
            assert col.dtype == e[k].dtype, k
            assert col.tolist() == e[k].tolist(), k
        assert _np(b.name_hash()).tolist() == e["name_hash"].tolist()
        assert b.names().to_bytes_list() == e["names"]
        assert _np(b.aligned_length()).tolist() == e["aligned_length"].tolist()
        assert _np(b.five_prime()).tolist() == e["five_prime"].tolist()
        assert _np(b.record_sizes()).tolist() == e["record_sizes"].tolist()
        for split in (0, 1):
            rec, start, end = b.blocks(split_deletions=bool(split))
            assert _np(rec).tolist() == e[f"blocks{split}_rec"].tolist()
            assert _np(start).tolist() == e[f"blocks{split}_start"].tolist()
            assert _np(end).tolist() == e[f"blocks{split}_end"].tolist()
        assert _np(b.base_at(e["base_rec"], e["base_pos"])).tolist() == e["base_at"].tolist()
        tags = b.tags(*TAGS)
        for t_name, t in zip(TAGS, tags):
            single = b.tag(t_name)
            p = f"tag_{t_name}_"
            for tt in (t, single):
                assert _np(tt.type).tolist() == e[p + "type"].tolist(), t_name
                assert _np(tt.offset).tolist() == e[p + "offset"].tolist(), t_name
                assert _np(tt.length).tolist() == e[p + "length"].tolist(), t_name
                assert _np(tt.value).tolist() == e[p + "value"].tolist(), t_name
            assert _np(t.hash()).tolist() == e[p + "hash"].tolist(), t_name
            code, ok = t.packed()
            assert _np(code).tolist() == e[p + "packed"].tolist(), t_name
            assert _np(ok).tolist() == e[p + "packed_ok"].astype(bool).tolist(), t_name
            assert t.strings().to_bytes_list() == e[p + "str"], t_name


def test_take_flags_and_unpack():
    (b,) = list(cubam_b200.read_bam(GOLDEN / "pairs.bam"))
    sel = b.has_flags(all_of=1, none_of=0x400)
    sub = b.take(sel)
    assert len(sub) == int(sel.sum())
    assert sub.data.data_ptr() == b.data.data_ptr()
    (b2,) = list(cubam_b200.read_bam(GOLDEN / "mixed_b65280.bam", chunk_bytes=1 << 22))
    code, ok = b2.tag("CB").packed()
    s = cubam_b200.unpack_acgt(code.view(torch.int64)[ok]).to_pylist()
    full = [x.decode() for x, k in zip(b2.tag("CB").strings().to_bytes_list(), _np(ok)) if k]
    assert s == full


def test_header_and_empty_bam():
    h = cubam_b200.BamHeader.read(GOLDEN / "empty.bam")
    g = meta()["header"]["empty.bam"]
    assert (h.text, h.names, h.lengths, h.size) == (g["text"], g["names"], g["lengths"], g["size"])
    assert h.lines("@PG") == g["pg"]
    assert list(cubam_b200.read_bam(GOLDEN / "empty.bam")) == []


def test_bgzf_chunks_match_reference():
    data = (GOLDEN / "text.raw").read_bytes()
    for key, sizes in meta()["bgzf"].items():
        name, chunk = key.split(":")
        chunks = list(cubam_b200.inflate_chunks(GOLDEN / name, chunk_bytes=int(chunk), piece=int(chunk) // 3 + 1))
        assert [int(c.numel()) for c in chunks] == sizes
        assert b"".join(_np(c).tobytes() for c in chunks) == data
        assert all(c.is_cuda for c in chunks)


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
        list(cubam_b200.inflate_chunks(GOLDEN / file, chunk_bytes=chunk))
    assert kind == "ValueError" and str(ei.value) == msg


def test_not_bgzf_empty_and_crc(tmp_path):
    p = tmp_path / "n.gz"
    p.write_bytes(b"hello world, not compressed" * 100)
    with pytest.raises(ValueError, match=meta()["errors"]["not_bgzf"][1]):
        list(cubam_b200.inflate_chunks(p, chunk_bytes=4096))
    p.write_bytes(G.EOF_BLOCK)
    assert sum(int(c.numel()) for c in cubam_b200.inflate_chunks(p, chunk_bytes=4096)) == 0
    bad = GOLDEN / "corrupt_bad_crc.gz"
    with pytest.raises(ValueError, match="CRC32"):
        list(cubam_b200.inflate_chunks(bad, chunk_bytes=8192))
    got = sum(int(c.numel()) for c in cubam_b200.inflate_chunks(bad, chunk_bytes=8192, check_crc=False))
    assert got == 50_000


def _payloads(seed: int):
    """Member contents of many shapes: text, random, runs, BAM-like, empty, 1 byte, 65536 bytes."""
    rng = random.Random(seed)
    nrng = np.random.default_rng(seed)
    out = [b"", b"x", b"\0" * 65536, bytes(nrng.integers(0, 256, 65280, dtype=np.uint8)), b"ab" * 32768]
    for _ in range(40):
        n = rng.choice([1, 2, 3, 100, 1000, 4095, 4096, 4097, 30000, 65280, 65535, 65536])
        kind = rng.randrange(5)
        if kind == 0:
            words = [bytes(rng.choices(b"ACGT\t\n0123456789:chr", k=rng.randint(1, 12))) for _ in range(50)]
            s = b"".join(rng.choice(words) for _ in range(n // 4 + 1))[:n]
        elif kind == 1:
            s = bytes(nrng.integers(0, 256, min(n, 65280), dtype=np.uint8))  # incompressible: fits a stored member
        elif kind == 2:
            s = bytes(nrng.integers(0, 4, n, dtype=np.uint8) * 17)
        elif kind == 3:
            base = bytes(nrng.integers(0, 256, rng.randint(1, 40000), dtype=np.uint8))
            s = (base * (n // max(len(base), 1) + 1))[:n]  # matches at long distances
        else:
            s = bytes(nrng.integers(2, 42, n, dtype=np.uint8))  # quality-like
        out.append(s)
    return out


# one member per warp, one member per lane, decode per lane + copy per warp (form 3 also with the copy
# kernel's groups of 32 and 128 units, 64 at 24 warps, with the decoder's 8-bit root tables, and with
# the two-range pipeline always and never)
FORMS = [1, 2, 3, "3/u1", "3/u4", "3/u2/w24", "3/r8", "3/p2", "3/p0"]
_FORM_PARAMS = {"u": G._lib.PARAM_COPY_UNITS, "w": G._lib.PARAM_COPY_WARPS, "r": G._lib.PARAM_DECODE_ROOT,
                "p": G._lib.PARAM_DECODE_PIPELINE}


class _Form:
    """An inflate form of FORMS with its launch parameters set, restored on exit."""

    def __init__(self, spec):
        parts = str(spec).split("/")
        self.form = int(parts[0])
        self.params = [(_FORM_PARAMS[x[0]], int(x[1:])) for x in parts[1:]]

    def __enter__(self):
        for key, v in self.params:
            assert G._lib.lib.cb_set_param(key, v) == 0
        return self.form

    def __exit__(self, *exc):
        for key, _ in self.params:
            G._lib.lib.cb_set_param(key, -1)


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize(
    ("level", "strategy"),
    [
        (6, zlib.Z_DEFAULT_STRATEGY),
        (1, zlib.Z_DEFAULT_STRATEGY),
        (9, zlib.Z_DEFAULT_STRATEGY),
        (0, zlib.Z_DEFAULT_STRATEGY),
        (6, zlib.Z_FIXED),
        (6, zlib.Z_HUFFMAN_ONLY),
        (6, zlib.Z_RLE),
        (6, zlib.Z_FILTERED),
    ],
)
def test_inflate_matches_zlib(tmp_path, level, strategy, form):
    payloads, members = [], []
    for p in _payloads(level * 10 + strategy):
        try:
            m = member(p, level, strategy)
        except OverflowError:  # even stored it does not fit: BGZF writers give a member at most 0xFF00 bytes
            p = p[:0xFF00]
            m = member(p, level, strategy)
        payloads.append(p)
        members.append(m)
    raw = b"".join(members)
    buf = torch.frombuffer(bytearray(raw), dtype=torch.uint8).cuda()
    jobs, s = G.scan_members(buf, True)
    assert s.status == 0 and s.n_members == len(payloads)
    assert s.total_out == sum(len(p) for p in payloads)
    out = torch.empty(int(s.total_out), dtype=torch.uint8, device="cuda")
    with _Form(form) as f:
        summ = G.inflate_jobs(jobs, int(s.n_jobs), out, True, form=f)
        G.check_inflate(summ)
    assert _np(out).tobytes() == b"".join(payloads)


@pytest.mark.parametrize("form", FORMS)
def test_inflate_output_alignment_and_offsets(form):
    """Members written at every output alignment (out_base offsets 0..17)."""
    payloads = _payloads(3)[:12]
    raw = b"".join(member(p) for p in payloads)
    buf = torch.frombuffer(bytearray(raw), dtype=torch.uint8).cuda()
    for shift in range(18):
        jobs, s = G.scan_members(buf, True, out_base=shift)
        out = torch.zeros(shift + int(s.total_out), dtype=torch.uint8, device="cuda")
        with _Form(form) as f:
            G.check_inflate(G.inflate_jobs(jobs, int(s.n_jobs), out, True, form=f))
        assert _np(out[shift:]).tobytes() == b"".join(payloads)
        assert not bool(out[:shift].any())


@pytest.mark.parametrize("form", FORMS)
def test_inflate_corrupt_members_are_errors(form):
    """Damaged members fail with the inflate or CRC status, never hang or overrun."""
    rng = random.Random(7)
    data = b"".join(bytes(rng.choices(b"ACGTN\t\n", k=200)) for _ in range(50))
    good = member(data)
    seen = set()
    for trial in range(200):
        m = bytearray(good)
        for _ in range(rng.randint(1, 4)):
            k = rng.randrange(18, len(m) - 8)
            m[k] ^= 1 << rng.randrange(8)
        buf = torch.frombuffer(bytearray(bytes(m) + G.EOF_BLOCK), dtype=torch.uint8).cuda()
        jobs, s = G.scan_members(buf, True)
        out = torch.empty(int(s.total_out), dtype=torch.uint8, device="cuda")
        with _Form(form) as f:
            st = int(G.read_struct(G.inflate_jobs(jobs, int(s.n_jobs), out, True, form=f),
                                   G._lib.InflateSummary).status)
        d = zlib.decompressobj(-15)
        try:
            z = d.decompress(bytes(m[18:-8]), len(data) + 1)
            zok = d.eof and len(z) == len(data)
        except zlib.error:
            zok = False
        if not zok:
            assert st in (G._lib.INFLATE, G._lib.CRC), trial
        else:
            assert st in (0, G._lib.CRC), trial
            if st == 0:
                assert _np(out).tobytes() == z
        seen.add(st)
    assert G._lib.INFLATE in seen


def test_inflate_many_members_all_forms_same_codes():
    """More members than the lane forms have lanes, so lanes take member after member; some members
    damaged.  Every form gives the payloads of the good members and the same per-job codes."""
    rng = random.Random(11)
    nrng = np.random.default_rng(11)
    n = int(G._lib.lib.cb_inflate_lane_slots()) + 3000
    assert n > 3000
    words = [bytes(rng.choices(b"ACGT\t\n0123456789:chrXY", k=rng.randint(1, 12))) for _ in range(200)]
    payloads, members, bad = [], [], set()
    for i in range(n):
        k = rng.choice([1, 2, 40, 300, 1000, 2500])
        p = b"".join(rng.choice(words) for _ in range(k // 4 + 1))[:k]
        if i % 97 == 5:
            p = bytes(nrng.integers(0, 256, k, dtype=np.uint8))  # stored blocks
        m = bytearray(member(p, rng.choice([1, 6, 9])))
        if i % 211 == 7 and len(m) > 40:
            m[18 + rng.randrange(len(m) - 26)] ^= 0x55
            bad.add(i)
        payloads.append(p)
        members.append(bytes(m))
    buf = torch.frombuffer(bytearray(b"".join(members) + G.EOF_BLOCK), dtype=torch.uint8).cuda()
    jobs, s = G.scan_members(buf, True)
    assert s.status == 0 and s.n_jobs == n
    results = []
    for form in FORMS:
        out = torch.zeros(int(s.total_out), dtype=torch.uint8, device="cuda")
        codes = torch.full((n,), 99, dtype=torch.int32, device="cuda")
        with _Form(form) as f:
            summ = G.read_struct(G.inflate_jobs(jobs, n, out, True, form=f, job_status=codes), G._lib.InflateSummary)
        codes = codes.cpu().numpy()
        assert (codes != 99).all()
        assert int(summ.n_bad) == int((codes != 0).sum())
        results.append((_np(out).tobytes(), codes))
    codes1 = results[0][1]
    for _, codes in results[1:]:
        assert (codes1 == codes).all()
    assert set(np.flatnonzero(codes1)) <= bad
    offs = np.cumsum([0] + [len(p) for p in payloads])
    good = np.flatnonzero(codes1 == 0)
    assert len(good) >= n - len(bad)
    for i in good[:: max(1, len(good) // 2000)].tolist() + good[-50:].tolist():
        for out, _ in results:
            assert out[offs[i]:offs[i + 1]] == payloads[i], i


def test_records_cross_members_and_chunks(tmp_path):
    """The oracle's batches on a BAM with small members and chunks (records split across both)."""
    raw = (GOLDEN / "mixed_b700.bam").read_bytes()
    for chunk in (3000, 7777, 50_000):
        exp = list(O.read_bam(raw, chunk, check_crc=True))
        got = list(cubam_b200.read_bam(GOLDEN / "mixed_b700.bam", chunk_bytes=chunk, piece=1000))
        assert [len(b) for b in got] == [len(b) for b in exp]
        for g, e in zip(got, exp):
            assert _np(g.data).tobytes() == e.data
            assert _np(g.offset).tolist() == e.offset.tolist()
            for k in O.FIELDS:
                assert _np(getattr(g, k)).tolist() == e.columns[k].tolist()


@pytest.mark.parametrize(("name", "chunk"), [("mixed_b700.bam", 50_000), ("pairs.bam", 1 << 20)])
def test_fused_record_pass_equals_the_separate_decoders(name, chunk):
    """decode(derived=True) gives the aligned lengths, name hashes and aligned blocks of the separate
    kernels, the blocks' counts from the same pass."""
    from golden_io import GOLDEN

    from cubam_b200.bam import RecordBatch

    for b in cubam_b200.read_bam(GOLDEN / name, chunk_bytes=chunk):
        f = RecordBatch.decode(b.data, b.offset, b.header, derived=True)
        for k in b.FIELDS:
            assert torch.equal(getattr(f, k), getattr(b, k)), k
        assert torch.equal(f.aligned_length(), b.aligned_length())
        assert torch.equal(f.name_hash().view(torch.int64), b.name_hash().view(torch.int64))
        for split in (False, True):
            assert f.__dict__["_derived"]["n_blocks_split" if split else "n_blocks"] is not None
            for x, y in zip(f.blocks(split), b.blocks(split)):
                assert torch.equal(x, y), split
        idx = torch.arange(0, len(b), 3, device="cuda")
        t = f.take(idx)
        assert torch.equal(t.aligned_length(), b.take(idx).aligned_length())
        for x, y in zip(t.blocks(True), b.take(idx).blocks(True)):
            assert torch.equal(x, y)


def test_too_many_member_candidates():
    """More than n/28 + 1024 member header matches in a chunk: the reference's "Too many candidates"
    error (src/cubam/bgzf.py:554, src/cubam/_kernels.py:671), as the oracle gives it, through the scan
    and through read_bam."""
    import tempfile

    from test_oracle import _fake_headers

    raw = _fake_headers(8000)
    with pytest.raises(ValueError, match="Too many candidates: the data is corrupt"):
        O.scan_members(raw, True)
    _, s = G.scan_members(torch.frombuffer(bytearray(raw), dtype=torch.uint8).cuda(), True)
    assert s.status == G._lib.TOO_MANY
    with pytest.raises(ValueError, match="Too many candidates: the data is corrupt"):
        G.raise_status(s.status, "scan")
    with tempfile.NamedTemporaryFile(suffix=".bam") as f:
        f.write(raw)
        f.flush()
        with pytest.raises(ValueError, match="Too many candidates: the data is corrupt"):
            list(cubam_b200.inflate_chunks(f.name))
