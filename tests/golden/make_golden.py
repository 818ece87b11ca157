"""Write the golden vectors under ``tests/golden/`` from the reference itself.

Run where the reference checkout exists (``$CUBAM_REFERENCE``, else a
directory ``reference`` beside this repository's root):
``python tests/golden/make_golden.py``.

1. The BAM/BGZF inputs are written by the reference's own fixture writer,
   ``tests/bamwriter.py`` (zlib level 6 raw deflate, ``bamwriter.py:15-29``),
   from seeded reads that cover every CIGAR operation, every aux type and a
   few malformed aux fields.
2. The expected outputs come from the reference's reader code
   (``src/cubam/bam.py``, ``src/cubam/bgzf.py`` and the kernels of
   ``src/cubam/_kernels.py`` compiled for the CPU), run through
   ``oracle/refrun.py``, for several chunk sizes; plus the reference's host
   helpers ``_fnv1a`` (``bam.py:164``), ``_pack_acgt`` (``cells.py:112``) and
   ``BamHeader.read`` (``bam.py:50``).
3. The writer's inputs are checked against the reference's outputs here (as
   ``tests/test_bam.py:60-80`` of the reference does) before anything is saved.
"""

from __future__ import annotations

import json
import random
import struct
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from oracle import refrun  # noqa: E402

TAGS = ("CB", "UB", "GN", "NM", "XS", "RG", "ZB", "xf", "NH", "XA", "Xc", "XC", "Xs", "Xi", "XI", "Xf", "XH", "ZZ", "QQ")
REFS = [("chr1", 1_000_000), ("chr2", 500_000), ("chrM", 16_569)]
OPS = "MIDNSHP=X"


def _bw():
    sys.path.insert(0, str(refrun.reference_tests_dir()))
    import bamwriter

    return bamwriter


def random_reads(bw, n: int, seed: int):
    """Seeded reads covering the CIGAR operations, aux types and odd records."""
    rng = random.Random(seed)

    class RawRead(bw.Read):
        """A read whose encoded bytes get ``extra`` aux bytes and Z->H retyping of ``XH``."""

        extra: bytes = b""

        def encode(self) -> bytes:
            b = super().encode()
            b = b.replace(b"XHZ", b"XHH")
            if self.extra:
                body = b[4:] + self.extra
                b = struct.pack("<i", len(body)) + body
            return b

    reads = []
    for i in range(n):
        ref = rng.randrange(len(REFS))
        kind = rng.random()
        parts = []
        if rng.random() < 0.1:
            parts.append(f"{rng.randint(1, 9)}H")
        if rng.random() < 0.3:
            parts.append(f"{rng.randint(1, 30)}S")
        m = rng.randint(10, 120)
        if kind < 0.4:
            parts.append(f"{m}M")
        elif kind < 0.6:
            parts += [f"{m // 2}M", f"{rng.randint(50, 5000)}N", f"{m - m // 2}M"]
        elif kind < 0.75:
            parts += [f"{m // 3}=", f"{rng.randint(1, 4)}X", f"{m // 3}M", f"{rng.randint(1, 3)}I", "3M"]
        elif kind < 0.9:
            parts += [f"{m // 2}M", f"{rng.randint(1, 5)}D", f"{m - m // 2}M", "1P", "2M"]
        else:
            parts += [f"{m}M", f"{rng.randint(1, 30)}S", f"{rng.randint(1, 30)}S"]
        if rng.random() < 0.25:
            parts.append(f"{rng.randint(1, 30)}S")
        if rng.random() < 0.1:
            parts.append(f"{rng.randint(1, 9)}H")
        cigar = "".join(parts)
        unmapped = rng.random() < 0.03
        tags = []
        if rng.random() < 0.9:
            bc = "".join(rng.choices("ACGT", k=rng.choice([16, 16, 16, 8, 24, 25])))
            tags.append(("CB", "Z", bc + rng.choice(["-1", "-1", "-12", "-123", "-1234", "", "-", "-x"])))
        if rng.random() < 0.8:
            tags.append(("UB", "Z", "".join(rng.choices("ACGTN", k=12))))
        if rng.random() < 0.5:
            tags.append(("GN", "Z", rng.choice(["ACTB", "GAPDH", "MT-CO1", "Gm12345", "", "LINC00115;AL669831.5"])))
        tags.append(("NM", "i", rng.randint(-3, 5)))
        tags.append(("XS", "C", rng.randint(0, 255)))
        if rng.random() < 0.3:
            sub = rng.choice("cCsSiIf")
            lo, hi = {"c": (-128, 127), "C": (0, 255), "s": (-32768, 32767), "S": (0, 65535),
                      "i": (-(2**31), 2**31 - 1), "I": (0, 2**32 - 1), "f": (-5, 5)}[sub]
            vals = [rng.uniform(lo, hi) if sub == "f" else rng.randint(lo, hi) for _ in range(rng.randint(0, 7))]
            tags.insert(0, ("ZB", "B", (sub, vals)))
        tags.append(("RG", "Z", f"group{rng.randint(0, 3)}"))
        if rng.random() < 0.4:
            tags.append(("xf", "i", rng.choice([0, 17, 25])))
            tags.append(("NH", "C", rng.randint(1, 4)))
        if rng.random() < 0.3:
            tags += [("XA", "A", rng.choice("ACGT+")), ("Xc", "c", rng.randint(-128, 127)),
                     ("XC", "C", rng.randint(0, 255)), ("Xs", "s", rng.randint(-32768, 32767)),
                     ("Xi", "i", rng.randint(-(2**31), 2**31 - 1)), ("XI", "I", rng.randint(0, 2**32 - 1)),
                     ("Xf", "f", rng.uniform(-1e3, 1e3)), ("XH", "Z", "".join(rng.choices("0123456789ABCDEF", k=8)))]
        name = "".join(rng.choices("ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789:_/#.|", k=rng.randint(1, 40)))
        r = RawRead(
            name=f"{name}{i}",
            flag=(4 if unmapped else 0) | rng.choice([0, 16, 99, 147, 83, 163, 1123, 256, 2048]),
            ref=-1 if unmapped and rng.random() < 0.5 else ref,
            pos=-1 if unmapped else rng.randrange(REFS[ref][1] - 6000),
            mapq=rng.choice([0, 1, 30, 60, 255]),
            cigar="" if unmapped else cigar,
            nref=rng.choice([-1, ref]),
            npos=rng.choice([-1, rng.randrange(REFS[ref][1])]),
            tlen=rng.randint(-1000, 1000),
            seq="".join(rng.choices("ACGTN=", k=rng.randint(0, 20))) if unmapped else "",
            qual=None,
            tags=tags,
        )
        if unmapped and r.ref < 0:
            r.nref = -1
        if not unmapped and rng.random() < 0.5:
            cig = bw.parse_cigar(cigar)
            n_seq = sum(k for op, k in cig if op in "MIS=X")
            r.seq = "".join(rng.choices("ACGTNRYKM", k=n_seq))
            r.qual = bytes(rng.randint(0, 41) for _ in range(n_seq))
        if rng.random() < 0.02:
            r.extra = b"ZQ?\x01"  # an aux field of unknown type: malformed
        elif rng.random() < 0.02:
            r.extra = b"ZQBi\xff\xff\x00\x00"  # a B array that runs past the record
        elif rng.random() < 0.02:
            r.extra = b"ZQ"  # 2 trailing bytes: the walk stops, no error
        reads.append(r)
    return sorted(reads, key=bw.sort_key)


def _strings_pack(lst):
    off = np.zeros(len(lst) + 1, np.int64)
    off[1:] = np.cumsum([len(x) for x in lst])
    return np.frombuffer(b"".join(lst), np.uint8).copy(), off


def _batch_arrays(cubam, b, rng: np.random.Generator, out: dict):
    """Every reader output of one batch, from the reference's own code, appended to ``out``'s lists."""
    n = len(b)

    def put(key, arr):
        out.setdefault(key, []).append(np.asarray(arr))

    put("n_records", [n])
    put("data_size", [int(b.data.size)])
    put("offset", b.offset.get())
    for k in cubam.RecordBatch.FIELDS:
        put(k, getattr(b, k).get())
    put("name_hash", b.name_hash().get())
    names = b.names()
    put("names_len", [len(x) for x in names])
    put("names_chars", np.frombuffer(b"".join(names), np.uint8))
    put("aligned_length", b.aligned_length().get())
    put("five_prime", b.five_prime().get())
    put("record_sizes", b.record_sizes().get())
    for split in (0, 1):
        rec, start, end = b.blocks(split_deletions=bool(split))
        put(f"blocks{split}_n", [int(rec.size)])
        put(f"blocks{split}_rec", rec.get())
        put(f"blocks{split}_start", start.get())
        put(f"blocks{split}_end", end.get())
    q = int(min(n, 64)) * 4
    rec = rng.integers(0, max(n, 1), q)
    refpos = b.pos.get()[rec].astype(np.int64) + rng.integers(-40, 200, q) if n else np.empty(0, np.int64)
    refpos = np.clip(refpos, -(2**31), 2**31 - 1).astype(np.int32)
    put("base_n", [q])
    put("base_rec", rec.astype(np.int64))
    put("base_pos", refpos)
    put("base_at", b.base_at(rec, refpos).get() if n else np.empty(0, np.int8))
    for name in TAGS:
        t = b.tag(name)
        tp = f"tag_{name}_"
        put(tp + "type", t.type.get())
        put(tp + "offset", t.offset.get())
        put(tp + "length", t.length.get())
        put(tp + "value", t.value.get())
        put(tp + "hash", t.hash().get())
        code, ok = t.packed()
        put(tp + "packed", code.get())
        put(tp + "packed_ok", ok.get())
        s = t.strings()
        put(tp + "str_len", [len(x) for x in s])
        put(tp + "str_chars", np.frombuffer(b"".join(s), np.uint8))


def bam_golden(cubam, bw, path: Path, chunks, reads, seed: int):
    """Golden npz files of one BAM, one per chunk size; checks the writer's inputs first.

    Each key holds the concatenation over batches; ``n_records``,
    ``blocks*_n`` and ``base_n`` give the per-batch lengths.
    """
    for chunk in chunks:
        out: dict = {}
        rng = np.random.default_rng(seed)
        batches = list(cubam.read_bam(path, chunk_bytes=chunk, piece=chunk // 2 + 1))
        for b in batches:
            _batch_arrays(cubam, b, rng, out)
        if reads is not None:
            got_pos = np.concatenate([b.pos.get() for b in batches]) if batches else np.empty(0)
            got_end = np.concatenate([b.end.get() for b in batches]) if batches else np.empty(0)
            got_names = sum((b.names() for b in batches), [])
            assert got_pos.tolist() == [r.pos for r in reads], path
            assert got_end.tolist() == [r.pos + (r.ref_len if r.cigar else 0) for r in reads], path
            assert got_names == [r.name.encode() for r in reads], path
        arrays = {k: np.concatenate(v) for k, v in out.items()}
        arrays["n_batches"] = np.int64(len(batches))
        np.savez_compressed(HERE / f"golden_{path.stem}_c{chunk}.npz", **arrays)


def text_data(n: int, seed: int) -> bytes:
    rng = random.Random(seed)
    words = [bytes(rng.choices(b"ACGT\t\n0123456789chrXY:", k=rng.randint(1, 30))) for _ in range(300)]
    out = bytearray()
    while len(out) < n:
        out += rng.choice(words)
    return bytes(out[:n])


def bgzf_golden(cubam, bw):
    """Inflated chunks and error outcomes of ``inflate_chunks`` on BGZF text."""
    data = text_data(120_000, 5)
    cases = {}
    for block, chunk in ((1000, 4096), (65280, 1 << 20), (300, 777)):
        name = f"text_b{block}.gz"
        p = HERE / name
        p.write_bytes(bw.bgzf(data, block))
        chunks = [c.get().tobytes() for c in cubam.inflate_chunks(p, chunk_bytes=chunk, piece=chunk // 3 + 1)]
        assert b"".join(chunks) == data
        cases[f"{name}:{chunk}"] = [len(c) for c in chunks]
    (HERE / "text.raw").write_bytes(data)
    errors = {}

    def outcome(raw: bytes, chunk: int):
        p = HERE / "_tmp.gz"
        p.write_bytes(raw)
        try:
            total = sum(int(c.size) for c in cubam.inflate_chunks(p, chunk_bytes=chunk))
            return ["ok", total]
        except (ValueError, RuntimeError) as e:
            return [type(e).__name__, str(e)]
        finally:
            p.unlink()

    small = bw.bgzf(data[:50_000], 1000)
    raw = bytearray(small)
    bsize = raw[16] + (raw[17] << 8) + 1
    errors["empty_file"] = outcome(bw.EOF_BLOCK, 4096)
    errors["truncated"] = outcome(bw.bgzf(data[:50_000], 1000, eof=False)[:-100], 8192)
    bt = bytearray(raw)
    bt[18] |= 0b110
    errors["bad_btype"] = outcome(bytes(bt), 8192)
    bi = bytearray(raw)
    bi[bsize - 4] ^= 0x01
    errors["bad_isize"] = outcome(bytes(bi), 8192)
    errors["not_bgzf"] = outcome(b"hello world, not compressed" * 100, 4096)
    bigi = bytearray(raw)
    bigi[bsize - 2] = 0x02  # ISIZE > 65536
    errors["isize_too_big"] = outcome(bytes(bigi), 8192)
    eofbad = bytearray(bw.EOF_BLOCK)
    eofbad[18] = 1  # empty member whose payload is not the empty fixed block
    errors["bad_empty_member"] = outcome(bytes(small) + bytes(eofbad), 8192)
    crc = bytearray(raw)
    crc[bsize - 8] ^= 0xFF  # CRC32 in the trailer: the reference does not check it
    errors["bad_crc_reference"] = outcome(bytes(crc), 8192)
    for name, raw_case in (("bad_btype", bt), ("bad_isize", bi), ("bad_crc", crc), ("isize_too_big", bigi)):
        (HERE / f"corrupt_{name}.gz").write_bytes(bytes(raw_case))
    (HERE / "corrupt_bad_empty_member.gz").write_bytes(bytes(small) + bytes(eofbad))
    (HERE / "truncated.gz").write_bytes(bw.bgzf(data[:50_000], 1000, eof=False)[:-100])
    return cases, errors


def main():
    cubam = refrun.load()
    if cubam is None:
        raise SystemExit("no reference checkout")
    bw = _bw()
    meta = {"bam": {}, "bgzf": {}, "errors": {}, "fnv1a": {}, "pack_acgt": {}, "header": {}}
    reads = random_reads(bw, 1500, seed=11)
    for block, chunks in ((700, (5000, 1 << 20)), (65280, (64 << 10, 20000))):
        p = bw.write_bam(HERE / f"mixed_b{block}.bam", REFS, reads, block=block)
        bam_golden(cubam, bw, p, chunks, reads, seed=block)
        meta["bam"][p.name] = list(chunks)
    longr = [bw.Read(f"long{i}", 0, 0, 1000 * i, 60, "20000M", -1, -1, 0) for i in range(12)]
    p = bw.write_bam(HERE / "long.bam", REFS, longr, block=4096)
    bam_golden(cubam, bw, p, (30_000,), longr, seed=1)
    meta["bam"][p.name] = [30_000]
    pairs = [bw.Read(f"pair{i}", 99, 0, 100 * i, 60, "50M", 0, 100 * i + 200, 250) for i in range(60)]
    pairs += [bw.Read(f"pair{i}", 147, 0, 100 * i + 200, 60, "50M", 0, 100 * i, -250) for i in range(60)]
    pairs.sort(key=bw.sort_key)
    p = bw.write_bam(HERE / "pairs.bam", REFS, pairs)
    bam_golden(cubam, bw, p, (1 << 20,), pairs, seed=2)
    meta["bam"][p.name] = [1 << 20]
    text = "@HD\tVN:1.6\tSO:coordinate\n@SQ\tSN:chr1\tLN:1000000\n@PG\tID:bwa\tPN:bwa\n"
    p = bw.write_bam(HERE / "empty.bam", REFS, [], text=text)
    bam_golden(cubam, bw, p, (4096,), [], seed=3)
    meta["bam"][p.name] = [4096]
    for name in ("mixed_b700.bam", "long.bam", "empty.bam"):
        h = cubam.BamHeader.read(HERE / name)
        meta["header"][name] = {"text": h.text, "names": h.names, "lengths": h.lengths, "size": h.size,
                                "sort_order": h.sort_order, "pg": h.lines("@PG")}
    meta["bgzf"], meta["errors"] = bgzf_golden(cubam, bw)
    from cubam.bam import _fnv1a
    from cubam.cells import _pack_acgt

    vals = ["", "A", "ACGT-1", "AAACCCAAGAAACACT-1", "read:1/2", "GENE_9", "ACGTN", "ACGT-123", "ACGT-1234",
            "A" * 24, "A" * 25, "ACGT-", "-1", "ACGT-x1"]
    meta["fnv1a"] = {v: int(x) for v, x in zip(vals, _fnv1a(vals))}
    meta["pack_acgt"] = {v: int(x) for v, x in zip(vals, _pack_acgt(vals))}
    (HERE / "golden.json").write_text(json.dumps(meta, indent=1, sort_keys=True))
    print("golden vectors written to", HERE)


if __name__ == "__main__":
    main()
