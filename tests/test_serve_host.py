"""Host logic of the serving loop (no GPU): the pool allocator, request slicing, Poisson requests."""

import numpy as np
import pytest

pytest.importorskip("torch")

from cubam_b200 import serve  # noqa: E402


def test_pool_allocator_first_fit_and_coalescing():
    a = serve.PoolAllocator(4096)
    x = a.alloc(1000)  # rounded to 1024
    y = a.alloc(1)  # 256
    z = a.alloc(2000)  # 2048
    assert (x, y, z) == (0, 1024, 1280)
    assert a.alloc(1024) is None and a.available() == 4096 - 1024 - 256 - 2048
    a.release(y, 1)
    assert a.alloc(200) == 1024  # first fit reuses the hole
    a.release(1024, 200)
    a.release(x, 1000)
    a.release(z, 2000)
    assert a.free == [(0, 4096)]


class _FakeIndex:
    def __init__(self, coff, first_rec):
        self.coff = np.asarray(coff, np.int64)
        self.first_rec = np.asarray(first_rec, np.int64)
        self.ucum = np.arange(len(coff), dtype=np.int64) * 65280
        self.cum_rec = np.arange(len(coff), dtype=np.int64) * 100


class _FakeFile:
    def __init__(self, coff, first_rec):
        self.index = _FakeIndex(coff, first_rec)

    boundaries = serve.ResidentFile.boundaries
    voff = serve.ResidentFile.voff
    member_of = serve.ResidentFile.member_of

    @property
    def n_members(self):
        return len(self.index.coff) - 1


def test_slices_cut_at_record_starts_within_the_limit():
    # 10 members of 1000 compressed bytes; no record starts in members 3 and 7
    coff = np.arange(11) * 1000
    first = [5, 0, 12, -1, 40, 0, 3, -1, 8, 1, 0]
    rf = _FakeFile(coff, first)
    req = serve.Request(0, rf.voff(0), rf.voff(10))
    req.m0, req.m1 = 0, 10
    for limit, want in [
        (2500, [(0, 2), (2, 4), (4, 6), (6, 8), (8, 10)]),
        (1000, [(0, 1), (1, 2), (2, 4), (4, 5), (5, 6), (6, 8), (8, 9), (9, 10)]),
        (100_000, [(0, 10)]),
    ]:
        assert serve.slice_request(rf, req, limit) == want
    with pytest.raises(ValueError):
        rf.member_of((3000 << 16) | 0)  # no record starts in member 3
    with pytest.raises(ValueError):
        rf.member_of((4000 << 16) | 41)  # not the first record of member 4
    assert rf.member_of(rf.voff(4)) == 4


def test_poisson_requests_are_record_aligned_and_ordered():
    coff = np.arange(201) * 30_000
    first = np.where(np.arange(201) % 7 == 3, -1, 17)
    first[-1] = 0
    rf = _FakeFile(coff, first)
    reqs = serve.poisson_requests([rf, rf], 300, rate=200.0, seed=1, min_bytes=64 << 10, max_bytes=4 << 20)
    t = [r.arrival for r in reqs]
    assert t == sorted(t) and 0.5 < t[-1] < 3.0  # ~1.5 s of arrivals at 200/s
    for r in reqs:
        m0, m1 = rf.member_of(r.voff_begin), rf.member_of(r.voff_end)
        assert m0 < m1
