"""Host logic of the serving loop's request deadline (no device work)."""

from cubam_b200 import _lib, serve


def _server(timeout):
    s = serve.Server.__new__(serve.Server)
    s.request_timeout = timeout
    s.timed_out = 0
    s.tags = ("CB",)
    s.alloc = serve.PoolAllocator(1 << 20)
    s.side_used = 0
    s.pending, s.active = [], []
    return s


def _admitted(s, rid, arrival, **kw):
    r = serve.Request(0, 0, 0, arrival=arrival, rid=rid)
    r._region_size, r.n_records = 4096, 10
    r._region = s.alloc.alloc(4096)
    s.side_used += r.n_records * serve.record_bytes(len(s.tags))
    for k, v in kw.items():
        setattr(r, k, v)
    s.active.append(r)
    return r


def test_deadline_rules():
    s = _server(1.0)
    waiting_late, waiting_new = serve.Request(0, 0, 0, arrival=0.0, rid=1), serve.Request(0, 0, 0, arrival=5.0, rid=2)
    s.pending += [waiting_late, waiting_new]
    idle = _admitted(s, 3, 0.0)  # admitted, nothing queued
    running = _admitted(s, 4, 0.0, _next=1, _inflight=1)  # a step holding it is queued
    last = _admitted(s, 5, 0.0, _last_launched=True, _inflight=1)  # its last slice is queued: served
    fresh = _admitted(s, 6, 1.5)
    out = []

    def finish(r):
        s._time_out(r, 2.0)
        out.append(r)

    s._expire(2.0, finish)
    assert [r.rid for r in out] == [1, 3]
    assert s.pending == [waiting_new] and idle not in s.active and idle._region == -1
    assert running._cancelled and running in s.active and running._region >= 0
    assert not last._cancelled and not fresh._cancelled
    for r in out:
        assert r.status == _lib.TIMEOUT and isinstance(r.error, TimeoutError) and r.done == 2.0
    assert s.timed_out == 2
    # the running one is freed by the loop once its queued step completes; the rest hold memory
    assert s.alloc.available() == (1 << 20) - 3 * 4096


def test_no_deadline():
    s = _server(None)
    s.pending.append(serve.Request(0, 0, 0, arrival=0.0))
    _admitted(s, 1, 0.0)
    s._expire(1e9, lambda r: (_ for _ in ()).throw(AssertionError("nothing expires")))
    assert len(s.pending) == 1 and len(s.active) == 1


def test_timeout_status_raises_timeout_error():
    import pytest

    from cubam_b200.bgzf import raise_status

    with pytest.raises(TimeoutError, match="deadline"):
        raise_status(_lib.TIMEOUT, "request 3")
    with pytest.raises(ValueError, match="Too many candidates"):
        raise_status(_lib.TOO_MANY, "scan")


# ---- step planning on a member index held on the host

def _fake_file(n_members=400, seed=3):
    """A resident file's index without its bytes: members of 15-30 KB compressed holding 65,280 inflated
    bytes; no record starts in about one member of ten (a long record crosses it)."""
    import numpy as np

    rng = np.random.default_rng(seed)
    csz = rng.integers(15_000, 30_000, n_members)
    coff = np.concatenate([[0], np.cumsum(csz)]).astype(np.int64)
    ucum = (np.arange(n_members + 1) * 65280).astype(np.int64)
    first = rng.integers(0, 300, n_members + 1).astype(np.int64)
    first[rng.random(n_members + 1) < 0.1] = -1
    first[0], first[n_members] = 0, 0
    counts = rng.integers(200, 260, n_members)
    cum = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    rf = serve.ResidentFile.__new__(serve.ResidentFile)
    rf.index = serve.MemberIndex(coff, ucum, first, cum, np.zeros((n_members, 4), np.int64))
    return rf


def _request(rf, a, b, rid=0):
    req = serve.Request(0, rf.voff(a), rf.voff(b), rid=rid)
    serve.plan_request(rf, req)
    return req


def test_slices_cover_the_request_at_record_starts():
    rf = _fake_file()
    ok = set(rf.boundaries().tolist())
    b = sorted(ok)
    for a_i, b_i in ((0, len(b) - 1), (5, 40), (100, 101), (3, 3)):
        req = _request(rf, b[a_i], b[b_i])
        sl = serve.slice_request(rf, req, 100_000)
        if req.m0 == req.m1:
            assert sl == []
            continue
        assert sl[0][0] == req.m0 and sl[-1][1] == req.m1
        for (x0, x1), (y0, _) in zip(sl, sl[1:]):
            assert x1 == y0
        for ma, mb in sl:
            assert mb in ok and mb > ma
            size = int(rf.index.coff[mb] - rf.index.coff[ma])
            # at most slice_bytes, unless no record start comes sooner
            nearer = [m for m in ok if ma < m < mb]
            assert size <= 100_000 or not nearer


def _planner(rf, step_bytes, short_bytes, small_bytes):
    s = serve.Server.__new__(serve.Server)
    s.files = [rf]
    s.long_step_bytes, s.short_step_bytes, s.small_bytes = step_bytes, short_bytes, small_bytes
    s.step_bytes = step_bytes
    s.slice_bytes = 100_000
    s.pending, s.active = [], []
    return s


def _admit(s, req):
    req._slices = serve.slice_request(s.files[0], req, s.slice_bytes)
    req._next = 0
    s.active.append(req)


def test_steps_keep_their_size_and_serve_the_oldest_first():
    rf = _fake_file()
    b = rf.boundaries()
    s = _planner(rf, step_bytes=1_000_000, short_bytes=300_000, small_bytes=50_000)
    big = [_request(rf, int(b[i]), int(b[i + 60]), rid=i) for i in (0, 100, 200)]
    for r in big:
        _admit(s, r)
    seen_slices = {r.rid: 0 for r in big}
    for _ in range(200):
        step = s._pick()
        if not step:
            break
        assert step[0].req is s.active[0] or step[0].req._next > 0  # the oldest request is served first
        total = sum(int(rf.index.coff[x.mb] - rf.index.coff[x.ma]) for x in step)
        assert total <= s.step_bytes or len(step) == 1
        assert s.step_bytes == 1_000_000  # no small request waits
        for x in step:
            seen_slices[x.req.rid] += 1
            if x.last:
                assert x.req._last_launched
        s.active = [r for r in s.active if not r._last_launched]
    assert not s.active  # every request got all its slices


def test_a_waiting_small_request_shortens_the_steps():
    rf = _fake_file()
    b = rf.boundaries()
    s = _planner(rf, step_bytes=1_000_000, short_bytes=300_000, small_bytes=50_000)
    _admit(s, _request(rf, int(b[0]), int(b[150]), rid=1))
    small = _request(rf, int(b[200]), int(b[201]), rid=2)
    assert small.compressed_bytes <= 50_000
    s.pending.append(small)  # arrived, not admitted yet
    step = s._pick()
    assert s.step_bytes == 300_000
    assert sum(int(rf.index.coff[x.mb] - rf.index.coff[x.ma]) for x in step) <= 300_000 or len(step) == 1
    s.pending.clear()
    _admit(s, small)
    step = s._pick()
    assert any(x.req is small for x in step)  # a started small request goes in the next step


def test_pool_allocator_never_overlaps_and_coalesces():
    import random

    rng = random.Random(5)
    pool = serve.PoolAllocator(1 << 24)
    live = {}
    for step in range(4000):
        if live and (rng.random() < 0.45 or pool.available() < (1 << 20)):
            off = rng.choice(list(live))
            pool.release(off, live.pop(off))
        else:
            n = rng.choice([1, 255, 256, 257, 4096, 100_000, 1 << 20])
            off = pool.alloc(n)
            if off is None:
                continue
            assert off % 256 == 0
            live[off] = n
        spans = sorted((o, o + ((n + 255) & ~255 or 256)) for o, n in live.items())
        for (a0, a1), (b0, _) in zip(spans, spans[1:]):
            assert a1 <= b0  # no two live ranges overlap
        assert all(a1 <= (1 << 24) for _, a1 in spans)
        assert pool.available() + sum(a1 - a0 for a0, a1 in spans) == 1 << 24
    for off, n in list(live.items()):
        pool.release(off, n)
    assert pool.free == [(0, 1 << 24)]
