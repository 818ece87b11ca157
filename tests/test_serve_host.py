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
