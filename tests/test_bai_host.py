"""BAI binning on the host: the torch reg2bin/reg2bins against the oracle's restatement of the spec."""

import random

import pytest

torch = pytest.importorskip("torch")

from cubam_b200 import bai  # noqa: E402
from oracle import bai_oracle  # noqa: E402


def test_reg2bin_matches_the_spec_restatement():
    rng = random.Random(3)
    beg, end = [], []
    for _ in range(5000):
        b = rng.randrange(0, 1 << 29)
        e = b + rng.choice([1, 2, 100, 16384, 70000, 1 << 20, 1 << 24]) if rng.random() < 0.9 else b + rng.randrange(1, 1 << 26)
        beg.append(b)
        end.append(min(e, 1 << 29))
    got = bai.reg2bin(torch.tensor(beg), torch.tensor(end)).tolist()
    assert got == [bai_oracle.reg2bin(b, e) for b, e in zip(beg, end)]
    # the leaf, level and root bins of the specification's layout
    assert bai_oracle.reg2bin(0, 1) == 4681 and bai_oracle.reg2bin(16384, 16385) == 4682
    assert bai_oracle.reg2bin(0, 1 << 29) == 0 and bai_oracle.reg2bin(0, 16385) == 585


def test_reg2bins_cover_the_bins_of_overlapping_records():
    rng = random.Random(4)
    for _ in range(300):
        b = rng.randrange(0, 1 << 28)
        e = b + rng.randrange(1, 1 << 22)
        bins = set(bai.reg2bins(b, e))
        assert bins == set(bai_oracle.reg2bins(b, e))
        for _ in range(20):  # any record overlapping [b, e) has its bin in the list
            rb = rng.randrange(max(0, b - (1 << 20)), e)
            re_ = max(rb + 1, rng.randrange(rb + 1, rb + (1 << 21)))
            if re_ > b:
                assert bai_oracle.reg2bin(rb, re_) in bins


def test_index_bytes_round_trip():
    idx = bai.BaiIndex([bai.RefIndex(), bai.RefIndex()], 7)
    import numpy as np

    idx.refs[0].bins[585] = np.array([[100, 200], [300, 400]], np.uint64)  # bin 585: [0, 131072)
    idx.refs[0].meta = (100, 400, 2, 0)
    idx.refs[0].lin = np.array([100, 250, 300], np.uint64)
    raw = idx.to_bytes()
    back = bai.BaiIndex.from_bytes(raw)
    assert back.to_bytes() == raw and back.n_no_coor == 7
    assert back.query(0, 0, 20000) == [(100, 200), (300, 400)]
    assert back.query(0, 20000, 30000) == [(300, 400)]  # the linear index drops chunks ending before 250
    assert back.query(0, 200000, 300000) == []  # no bin of the region holds a chunk
    assert back.query(1, 0, 10) == []
