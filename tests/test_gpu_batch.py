"""The batched decoder: one inflate launch for the members of many files, and its graph-replayed plan.

An uneven batch in the shape of the 64-file workload (GEX or ATAC records, zlib levels 1..9 per
member, 2% stored members), scaled down: every file's records, columns and tags from
``decode_many`` equal the C oracle's (zlib + struct decoding on the host), and the plan's eager
launches in both inflate forms and its CUDA-graph replays equal ``decode_many``.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

import cubam_b200  # noqa: E402
from cubam_b200 import batch, synth  # noqa: E402
from oracle import cpu_oracle  # noqa: E402

TAGS = ("CB", "UB", "GN")
FIELDS = cpu_oracle.FIELDS


@pytest.fixture(scope="module")
def uneven(tmp_path_factory):
    d = tmp_path_factory.mktemp("uneven")
    out = []
    for cfg in synth.uneven_files(scale=0.002)[:24]:
        p = d / f"{cfg.name}.bam"
        synth.write_bam(p, cfg)
        raw = p.read_bytes()
        out.append((raw, batch.load_compressed(p), cubam_b200.BamHeader.read(p)))
    return out


def _cpu(a):
    return a.cpu().numpy()


def _same(res, ref):
    """Two DecodedFile results are equal, byte for byte."""
    assert len(res) == len(ref)
    assert torch.equal(res.data, ref.data)
    assert torch.equal(res.offset, ref.offset)
    for f in FIELDS:
        assert torch.equal(res.columns[f], ref.columns[f]), f
    for t in TAGS:
        a, b = res.tags[t], ref.tags[t]
        for x in ("type", "offset", "length", "value"):
            assert torch.equal(getattr(a, x), getattr(b, x)), (t, x)


def test_decode_many_matches_cpu_oracle(uneven):
    files = [(comp, hdr) for _, comp, hdr in uneven]
    got = batch.decode_many(files, tags=TAGS)
    for (raw, _, _), res in zip(uneven, got):
        want = cpu_oracle.decode_file(raw, tags=TAGS)
        assert res.n_members == want.n_members
        assert _cpu(res.data).tobytes() == want.data.tobytes()
        assert np.array_equal(_cpu(res.offset), want.offset)
        for f in FIELDS:
            assert np.array_equal(_cpu(res.columns[f]), want.columns[f]), f
        for t in TAGS:
            ty, vo, vl, iv, _ = want.tags[t]
            tag = res.tags[t]
            assert np.array_equal(_cpu(tag.type), ty), t
            assert np.array_equal(_cpu(tag.offset), vo), t
            assert np.array_equal(_cpu(tag.length), vl), t
            assert np.array_equal(_cpu(tag.value), iv), t


def test_batch_plan_forms_and_graph_replay(uneven):
    files = [(comp, hdr) for _, comp, hdr in uneven]
    ref = batch.decode_many(files, tags=TAGS)
    plan = batch.BatchPlan(files, tags=TAGS)
    assert plan.form in (1, 2, 3) and set(plan.tuning["ms"]["inflate_form"]) == {"1", "2", "3"}
    for form in (1, 2, 3):
        for r in plan.results:  # nothing stale can pass
            r.data.fill_(0)
            for c in r.columns.values():
                c.fill_(0)
        plan.launch(form)
        torch.cuda.synchronize()
        plan.check()
        for a, b in zip(plan.results, ref):
            _same(a, b)
    plan.capture()
    for _ in range(2):
        plan.out.fill_(0)
        plan.replay()
        torch.cuda.synchronize()
        plan.check()
        for a, b in zip(plan.results, ref):
            _same(a, b)
    assert plan.launches_per_run() > len(files)


def test_native_batch_matches_decode_many(uneven):
    """The batch planned and run by the library (cb_batch_*): results equal decode_many's, again after
    eager runs and after graph replays that rewrite them in place."""
    files = [(comp, hdr) for _, comp, hdr in uneven]
    ref = batch.decode_many(files, tags=TAGS)
    nb = batch.NativeBatch(files, tags=TAGS)
    assert nb.form in (1, 2, 3)
    for res, r in zip(nb.results, ref):
        _same(res, r)
        assert res.n_members == r.n_members and res.inflated_bytes == r.inflated_bytes
    for res in nb.results:
        res.columns["pos"].fill_(-7)
        res.offset.fill_(-1)
    nb.run()
    nb.check()
    for res, r in zip(nb.results, ref):
        _same(res, r)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        nb.capture()
        for res in nb.results:
            res.columns["pos"].fill_(-7)
            res.tags["CB"].offset.fill_(0)
        for _ in range(2):
            nb.run()
        nb.check()
    torch.cuda.synchronize()
    for res, r in zip(nb.results, ref):
        _same(res, r)
    nb.close()


def test_native_batch_errors(uneven):
    _, comp, hdr = uneven[0]
    with pytest.raises(ValueError, match="Truncated BGZF file"):
        batch.NativeBatch([(comp[: comp.numel() - 100].clone(), hdr)], tags=TAGS)
    bad = comp.clone()
    bad[30:60] = 0  # inside the first member's DEFLATE data
    with pytest.raises(ValueError, match="Corrupt BGZF block|No valid block"):
        batch.NativeBatch([(bad, hdr)], tags=TAGS)
