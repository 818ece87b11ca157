"""GPU parity on the benchmark workloads themselves, against the C oracle.

- the small workload exactly as specified (100,000 single-end 90 bp records, one 1 Mb reference,
  uniform qualities 2..41, CB from 1,000 barcodes, UB random; seed 0), read by ``read_bam`` at
  three chunk sizes that split records across members and chunks: every batch's record bytes,
  offsets, the 11 fixed columns, the CB/UB tags, their FNV-1a hashes and packed codes, and the
  read-name hashes;
- GEX- and ATAC-shaped files of 1,000,000 records (the shapes of the 50M-record and 100M-record
  workloads, fewer records), read by ``read_bam`` in 32 MB chunks and by the batched whole-file
  decoder: columns and CB/UB/GN tags.

The oracle is ``oracle/cpu_decoder.c`` (zlib inflate, record chain, columns, tags on the host).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

import cubam_b200  # noqa: E402
from cubam_b200 import batch, synth  # noqa: E402
from oracle import bam_oracle as O  # noqa: E402
from oracle import cpu_oracle  # noqa: E402

FIELDS = cubam_b200.RecordBatch.FIELDS


def _np(t):
    return t.cpu().numpy()


@pytest.fixture(scope="module")
def small(tmp_path_factory):
    path = tmp_path_factory.mktemp("cfg") / "small.bam"
    synth.write_bam(path, "small")
    raw = path.read_bytes()
    return path, cpu_oracle.decode_file(raw, tags=("CB", "UB"))


def _check_batches(batches, ref, tags, packed=False):
    """The batches of ``read_bam``, in order, equal the oracle's decode of the whole file."""
    k = 0
    for b in batches:
        n = len(b)
        off = _np(b.offset)
        roff = ref.offset[k : k + n]
        # the same records: positions relative to the batch's first record, and the record bytes
        assert (off - off[0]).tolist() == (roff - roff[0]).tolist()
        end = int(roff[-1]) + int(np.frombuffer(ref.data[int(roff[-1]) : int(roff[-1]) + 4], "<u4")[0]) + 4
        assert _np(b.data[int(off[0]) : int(off[0]) + end - int(roff[0])]).tobytes() == ref.data[int(roff[0]) : end].tobytes()
        for f in FIELDS:
            assert _np(getattr(b, f)).tolist() == ref.columns[f][k : k + n].tolist(), f
        assert _np(b.name_hash()).tolist() == ref.name_hash[k : k + n].tolist()
        for name, t in zip(tags, b.tags(*tags)):
            ty, vo, vl, iv, th = (x[k : k + n] for x in ref.tags[name])
            assert _np(t.type).tolist() == ty.tolist(), name
            # a present tag's offset within its record; a missing one has offset 0 in both
            present = (ty != 0) & (ty != 255)
            goff = _np(t.offset)
            assert np.where(present, goff - off, goff).tolist() == np.where(present, vo - roff, vo).tolist(), name
            assert _np(t.length).tolist() == vl.tolist(), name
            assert _np(t.value).tolist() == iv.tolist(), name
            assert _np(t.hash()).tolist() == th.tolist(), name
            if packed:
                codes, ok = t.packed()
                ecodes, eok = O.tag_packed(ref.data.tobytes(), ty, vo, vl)
                assert _np(codes).tolist() == np.asarray(ecodes).tolist(), name
                assert _np(ok).tolist() == np.asarray(eok, dtype=bool).tolist(), name
        k += n
    assert k == len(ref.offset)


@pytest.mark.parametrize("chunk", [1 << 20, 3_000_017, 64 << 20])
def test_small_workload_read_bam(small, chunk):
    path, ref = small
    assert len(ref.offset) == 100_000
    _check_batches(cubam_b200.read_bam(path, chunk_bytes=chunk), ref, ("CB", "UB"), packed=True)


@pytest.fixture(scope="module", params=["gex", "atac"])
def shaped(request, tmp_path_factory):
    path = tmp_path_factory.mktemp("cfg") / f"{request.param}_1m.bam"
    synth.write_bam(path, request.param, n_records=1_000_000)
    return path, cpu_oracle.decode_file(path.read_bytes(), tags=("CB", "UB", "GN"))


def test_shaped_workloads_read_bam(shaped):
    path, ref = shaped
    assert len(ref.offset) == 1_000_000
    _check_batches(cubam_b200.read_bam(path, chunk_bytes=32 << 20), ref, ("CB", "UB", "GN"))


def test_shaped_workloads_batched(shaped):
    path, ref = shaped
    comp = batch.load_compressed(path)
    d = batch.decode_resident(comp, cubam_b200.BamHeader.read(path), tags=("CB", "UB", "GN"))
    assert _np(d.offset).tolist() == ref.offset.tolist()
    for f in FIELDS:
        assert _np(d.columns[f]).tolist() == ref.columns[f].tolist(), f
    for name, t in d.tags.items():
        ty, vo, vl, iv, _ = ref.tags[name]
        assert _np(t.type).tolist() == ty.tolist(), name
        assert _np(t.offset).tolist() == vo.tolist(), name
        assert _np(t.length).tolist() == vl.tolist(), name
        assert _np(t.value).tolist() == iv.tolist(), name


@pytest.mark.parametrize("tile", [2048, 8192, 65536])
def test_chain_tiles_give_the_oracle_offsets(shaped, tile):
    """The record chain at each tile size (a tile walked by a warp through 8 KB windows) gives the
    oracle's record offsets and the same columns."""
    from cubam_b200 import _lib

    path, ref = shaped
    comp = batch.load_compressed(path)
    assert _lib.lib.cb_set_param(_lib.PARAM_CHAIN_TILE, tile) == 0
    try:
        d = batch.decode_resident(comp, cubam_b200.BamHeader.read(path), tags=())
    finally:
        _lib.lib.cb_set_param(_lib.PARAM_CHAIN_TILE, -1)
    assert _np(d.offset).tolist() == ref.offset.tolist()
    assert _np(d.columns["pos"]).tolist() == ref.columns["pos"].tolist()


def _long_records_bam(path, n=3000, seed=12):
    """A BAM whose records are mostly ordinary (90 bp) but include long ones: reads of 5-40 kb, CIGARs
    of up to 600 operations, names up to 200 characters, a 12 KB aux string and B arrays -- records
    larger than the record kernels' shared-memory windows (8-12 KB), spanning many BGZF members."""
    import struct
    import zlib

    from cubam_b200.bgzf import EOF_BLOCK

    rng = np.random.default_rng(seed)
    refs = [(b"chr1", 50_000_000), (b"chr2", 40_000_000)]
    text = b"@HD\tVN:1.6\tSO:coordinate\n" + b"".join(b"@SQ\tSN:%s\tLN:%d\n" % r for r in refs)
    head = b"BAM\1" + struct.pack("<i", len(text)) + text + struct.pack("<i", len(refs))
    head += b"".join(struct.pack("<i", len(nm) + 1) + nm + b"\0" + struct.pack("<i", ln) for nm, ln in refs)
    recs, pos = [], 1000
    for i in range(n):
        pos += int(rng.integers(0, 400))
        long = rng.random() < 0.05
        if long:  # a long read with many operations: M, I, D, N, S
            ops, l_seq = [], 0
            for _ in range(int(rng.integers(50, 600))):
                op = int(rng.choice([0, 0, 0, 1, 2, 3]))
                ln = int(rng.integers(1, 80))
                ops.append((op, ln))
                l_seq += ln if op in (0, 1) else 0
            ops = [(4, 12)] + ops + [(4, 7)]
            l_seq += 19
            name = b"L" + bytes(rng.integers(65, 91, int(rng.integers(20, 200))).astype(np.uint8))
        else:
            ops, l_seq = [(0, 90)], 90
            name = b"r%d" % i
        rlen = sum(ln for op, ln in ops if op in (0, 2, 3, 7, 8))
        cig = b"".join(struct.pack("<I", (ln << 4) | op) for op, ln in ops)
        seq = bytes(rng.integers(0, 256, (l_seq + 1) // 2).astype(np.uint8))
        qual = bytes(rng.integers(2, 42, l_seq).astype(np.uint8))
        aux = b"CBZ" + b"ACGTACGTACGTACGT-1\0" + b"UBZ" + bytes(rng.choice(list(b"ACGT"), 10).astype(np.uint8)) + b"\0"
        if long:
            aux += b"XSZ" + bytes(rng.integers(33, 127, 12_000).astype(np.uint8)) + b"\0"
            aux += b"XBBi" + struct.pack("<i", 300) + struct.pack("<300i", *rng.integers(-9, 9, 300))
        aux += b"GNZ" + b"GENE%d\0" % (i % 50) + b"NHi" + struct.pack("<i", 1)
        body = struct.pack("<iiBBHHHIiii", 0, pos, len(name) + 1, 60, O.reg2bin(pos, pos + max(rlen, 1)), len(ops),
                           16 if i % 3 == 0 else 0, l_seq, -1, -1, 0)
        body += name + b"\0" + cig + seq + qual + aux
        recs.append(struct.pack("<i", len(body)) + body)
    blob = head + b"".join(recs)
    members = []
    for a in range(0, len(blob), 0xFF00):
        c = zlib.compressobj(6, zlib.DEFLATED, -15)
        payload = c.compress(blob[a : a + 0xFF00]) + c.flush()
        bsize = 18 + len(payload) + 8
        members.append(b"\x1f\x8b\x08\x04\0\0\0\0\0\xff\x06\0BC\x02\0" + struct.pack("<H", bsize - 1) + payload
                       + struct.pack("<II", zlib.crc32(blob[a : a + 0xFF00]), len(blob[a : a + 0xFF00])))
    path.write_bytes(b"".join(members) + EOF_BLOCK)
    return path


@pytest.fixture(scope="module")
def long_records(tmp_path_factory):
    path = _long_records_bam(tmp_path_factory.mktemp("long") / "long.bam")
    return path, cpu_oracle.decode_file(path.read_bytes(), tags=("CB", "UB", "GN"))


@pytest.mark.parametrize("chunk", [300_000, 4 << 20])
def test_long_records_read_bam(long_records, chunk):
    path, ref = long_records
    assert len(ref.offset) == 3000
    _check_batches(cubam_b200.read_bam(path, chunk_bytes=chunk), ref, ("CB", "UB", "GN"))


@pytest.mark.parametrize("tile", [2048, 65536])
def test_long_records_batched(long_records, tile):
    """Records longer than a chain tile (tiles with no record start) and than the staged windows."""
    from cubam_b200 import _lib

    path, ref = long_records
    comp = batch.load_compressed(path)
    assert _lib.lib.cb_set_param(_lib.PARAM_CHAIN_TILE, tile) == 0
    try:
        d = batch.decode_resident(comp, cubam_b200.BamHeader.read(path), tags=("CB", "UB", "GN"))
    finally:
        _lib.lib.cb_set_param(_lib.PARAM_CHAIN_TILE, -1)
    assert _np(d.offset).tolist() == ref.offset.tolist()
    for f in FIELDS:
        assert _np(d.columns[f]).tolist() == ref.columns[f].tolist(), f
    for name, t in d.tags.items():
        ty, vo, vl, iv, _ = ref.tags[name]
        assert _np(t.type).tolist() == ty.tolist(), name
        assert _np(t.offset).tolist() == vo.tolist(), name
        assert _np(t.length).tolist() == vl.tolist(), name
