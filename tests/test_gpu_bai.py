"""BAI index built on the device, and region fetches through it.

- The index bytes equal the oracle's restatement of the specification's index
  (oracle/bai_oracle.py) over the C oracle's decoded records and their virtual offsets.
- A region fetch gives exactly the records of the whole-file decode that overlap the region
  (same columns, tags and record offsets), over random regions of GEX and ATAC files.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from cubam_b200 import bai, batch, serve, synth  # noqa: E402
from cubam_b200.synth import Config  # noqa: E402
from oracle import bai_oracle, bam_oracle, cpu_oracle  # noqa: E402

TAGS = ("CB", "UB", "GN")
FIELDS = cpu_oracle.FIELDS


@pytest.fixture(scope="module")
def files(tmp_path_factory):
    d = tmp_path_factory.mktemp("bai")
    out = []
    for c in (Config("g", 1, 120_000, 51), Config("a", 2, 160_000, 52, n_barcodes=10_000),
              Config("m", 1, 40_000, 53, level=-1, stored_frac=0.05)):
        p = d / f"{c.name}.bam"
        synth.write_bam(p, c)
        out.append((p.read_bytes(), serve.ResidentFile.load(p)))
    return out


def _oracle_voffs(raw: bytes, starts: np.ndarray):
    """Virtual offsets of records (absolute inflated offsets), and of their ends, on the host."""
    offs, bsize, isize, _ = bam_oracle.scan_members(raw, True)
    data = np.flatnonzero(np.asarray(isize) > 0)
    coff = np.asarray(offs, np.int64)[data]
    ucum = np.concatenate([[0], np.cumsum(np.asarray(isize, np.int64))])[data]
    end = int(coff[-1] + np.asarray(bsize, np.int64)[data][-1])
    m = np.searchsorted(ucum, starts, side="right") - 1
    voff = (coff[m] << 16) | (starts - ucum[m])
    nxt = np.append(voff[1:], end << 16)
    return voff, nxt


def test_index_bytes_match_the_oracle(files):
    for raw, rf in files:
        want = cpu_oracle.decode_file(raw, tags=())
        starts = want.offset + rf.header.size
        voff, nxt = _oracle_voffs(raw, starts)
        c = want.columns
        ref_bytes = bai_oracle.build(len(rf.header.names), c["ref"], c["pos"], c["end"], c["flag"], voff, nxt)
        idx = bai.build(rf)
        got = idx.to_bytes()
        assert got == ref_bytes
        assert bai.BaiIndex.from_bytes(got).to_bytes() == got


def test_region_fetch_equals_the_whole_file_filtered(files):
    rng = np.random.default_rng(8)
    for raw, rf in files:
        idx = bai.build(rf)
        whole = batch.decode_many([(rf.comp, rf.header)], tags=TAGS)[0]
        W = {k: whole.columns[k].cpu().numpy() for k in FIELDS}
        woff = whole.offset.cpu().numpy()
        wt = {t: {x: getattr(whole.tags[t], x).cpu().numpy() for x in ("type", "offset", "length", "value")}
              for t in TAGS}
        used = np.unique(W["ref"][W["ref"] >= 0])
        regions = [(int(used[0]), 0, 1 << 29), (int(used[0]), 5, 6)]
        for _ in range(30):
            r = int(rng.choice(used))
            pr = W["pos"][W["ref"] == r]
            beg = int(rng.integers(max(int(pr.min()) - 100_000, 0), int(pr.max()) + 10))
            regions.append((r, beg, beg + int(np.exp(rng.uniform(0, np.log(5e6))))))
        for r, beg, end in regions:
            got = bai.fetch(rf, idx, r, beg, end, tags=TAGS)
            sel = np.flatnonzero(bai_oracle.overlaps(W["ref"], W["pos"], W["end"], r, beg, end))
            assert len(got) == len(sel), (r, beg, end)
            if not len(sel):
                continue
            go = got.offset.cpu().numpy()
            data_start = int(woff[sel[0]] - go[0])  # where the fetched bytes start in the file's records
            assert np.array_equal(go + data_start, woff[sel])
            for k in FIELDS:
                assert np.array_equal(got.columns[k].cpu().numpy(), W[k][sel]), k
            for t in TAGS:
                T = got.tags[t]
                ty = wt[t]["type"][sel]
                present = (ty != 0) & (ty != 255)
                assert np.array_equal(T.type.cpu().numpy(), ty)
                assert np.array_equal(T.length.cpu().numpy(), wt[t]["length"][sel])
                assert np.array_equal(T.value.cpu().numpy(), wt[t]["value"][sel])
                o = T.offset.cpu().numpy()
                assert np.array_equal(np.where(present, o + data_start, o), wt[t]["offset"][sel])

