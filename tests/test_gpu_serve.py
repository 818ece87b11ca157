"""The serving loop: each request's records, columns and tags are the same decoded alone, served in a
mix with others (split into slices, sharing steps and inflate launches), and cut from the whole
file's decode."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from cubam_b200 import batch, serve, synth  # noqa: E402
from cubam_b200.synth import Config  # noqa: E402

TAGS = ("CB", "UB", "GN")
FIELDS = ("ref", "pos", "end", "mapq", "flag", "nref", "npos", "tlen", "l_seq", "clip_left", "clip_right")


@pytest.fixture(scope="module")
def files(tmp_path_factory):
    d = tmp_path_factory.mktemp("serve")
    cfgs = [Config("g", 1, 60_000, 41), Config("a", 2, 90_000, 42, n_barcodes=10_000),
            Config("m", 1, 25_000, 43, level=-1, stored_frac=0.05)]
    out = []
    for c in cfgs:
        p = d / f"{c.name}.bam"
        synth.write_bam(p, c)
        out.append(serve.ResidentFile.load(p))
    return out


def _host(res):
    return {
        "data": res.data.cpu().numpy().tobytes(),
        "offset": res.offset.cpu().numpy(),
        **{f: res.columns[f].cpu().numpy() for f in FIELDS},
        **{f"{t}.{x}": getattr(res.tags[t], x).cpu().numpy() for t in TAGS for x in ("type", "offset", "length", "value")},
    }


def _equal(a, b):
    assert a.keys() == b.keys()
    for k in a:
        if k == "data":
            assert a[k] == b[k]
        else:
            assert np.array_equal(a[k], b[k]), k


def _ranges(rf, rng, n):
    ok = rf.boundaries()
    out = [(int(ok[0]), int(ok[-1])), (int(ok[0]), int(ok[0])), (int(ok[-2]), int(ok[-1]))]
    while len(out) < n:
        a, b = sorted(int(x) for x in rng.choice(ok, 2, replace=False))
        out.append((a, b))
    return out


def test_index_matches_the_whole_file(files):
    for rf in files:
        whole = batch.decode_many([(rf.comp, rf.header)], tags=())[0]
        ix = rf.index
        assert int(ix.cum_rec[-1]) == len(whole)
        starts = whole.offset.cpu().numpy() + rf.header.size
        for m in rf.boundaries()[:-1]:
            k = int(ix.cum_rec[m])
            assert starts[k] == ix.ucum[m] + ix.first_rec[m]
            assert rf.member_of(rf.voff(int(m))) == m


def test_requests_alone_match_the_whole_file(files):
    rng = np.random.default_rng(5)
    for rf in files:
        whole = _host(batch.decode_many([(rf.comp, rf.header)], tags=TAGS)[0])
        for a, b in _ranges(rf, rng, 12):
            req = serve.Request(0, rf.voff(a), rf.voff(b))
            got = _host(serve.decode_alone(rf, req, tags=TAGS))
            ix = rf.index
            r0, r1 = int(ix.cum_rec[a]), int(ix.cum_rec[b])
            assert len(got["offset"]) == r1 - r0 == req.n_records
            shift = int(ix.ucum[a] + ix.first_rec[a]) - rf.header.size  # request data start in the whole file
            w0 = shift
            assert got["data"] == whole["data"][w0 : w0 + req.inflated_bytes]
            assert np.array_equal(got["offset"], whole["offset"][r0:r1] - shift)
            for f in FIELDS:
                assert np.array_equal(got[f], whole[f][r0:r1]), f
            for t in TAGS:
                ty = whole[f"{t}.type"][r0:r1]
                present = (ty != 0) & (ty != 255)  # a missing or malformed tag has offset 0
                want = np.where(present, whole[f"{t}.offset"][r0:r1] - shift, whole[f"{t}.offset"][r0:r1])
                assert np.array_equal(got[f"{t}.offset"], want), t
                for x in ("type", "length", "value"):
                    assert np.array_equal(got[f"{t}.{x}"], whole[f"{t}.{x}"][r0:r1]), (t, x)


def test_served_in_a_mix_equals_alone(files):
    rng = np.random.default_rng(6)
    reqs = []
    for f, rf in enumerate(files):
        for a, b in _ranges(rf, rng, 14):
            reqs.append(serve.Request(f, rf.voff(a), rf.voff(b), arrival=float(rng.uniform(0, 0.05)), rid=len(reqs)))
    alone = {r.rid: _host(serve.decode_alone(files[r.file], serve.Request(r.file, r.voff_begin, r.voff_end), TAGS))
             for r in reqs}
    got = {}

    def on_done(r):
        got[r.rid] = _host(r.result)

    # a small budget and small slices and steps: requests wait for memory, split into several
    # slices, and share steps with others
    server = serve.Server(files, budget_bytes=48 << 20, step_bytes=1 << 20, slice_bytes=256 << 10, tags=TAGS)
    done = server.run(reqs, on_done=on_done)
    assert len(done) == len(reqs) and set(got) == {r.rid for r in reqs}
    assert server.steps > len(reqs) // 2
    assert max(n for n, _ in server.step_log) > 1  # steps held slices of several requests
    assert any(len(serve.slice_request(files[r.file], r, 256 << 10)) > 2 for r in reqs)
    assert server.alloc.free == [(0, server.pool_bytes)] and server.side_used == 0
    for r in reqs:
        _equal(got[r.rid], alone[r.rid])
        assert r.done is not None and r.done >= r.arrival
    lat = serve.latency_summary(done)
    assert lat["all_ms"]["n"] == len(reqs)


def test_request_timeout(files):
    """With a deadline of 0 s every request times out (those not started at once, those started after
    their queued steps), the rest of the loop carries on, and all memory comes back; without one the
    same requests are all served."""
    rng = np.random.default_rng(9)
    reqs = []
    for f, rf in enumerate(files):
        for a, b in _ranges(rf, rng, 6):
            reqs.append(serve.Request(f, rf.voff(a), rf.voff(b), arrival=0.0, rid=len(reqs)))
    seen = []
    server = serve.Server(files, budget_bytes=48 << 20, step_bytes=1 << 20, slice_bytes=256 << 10, tags=TAGS,
                          request_timeout=0.0)
    done = server.run(reqs, on_done=seen.append)
    assert len(done) == len(reqs) == len(seen)
    late = [r for r in done if r.status == serve._lib.TIMEOUT]
    assert late and server.timed_out == len(late)
    for r in late:
        assert r.result is None and isinstance(r.error, TimeoutError)
    for r in done:
        assert r.status in (0, serve._lib.TIMEOUT)
    assert server.alloc.free == [(0, server.pool_bytes)] and server.side_used == 0 and not server.active

    again = [serve.Request(r.file, r.voff_begin, r.voff_end, rid=r.rid) for r in reqs]
    server = serve.Server(files, budget_bytes=48 << 20, step_bytes=1 << 20, slice_bytes=256 << 10, tags=TAGS,
                          request_timeout=60.0)
    done = server.run(again)
    assert server.timed_out == 0 and all(r.status == 0 for r in done) and len(done) == len(again)
