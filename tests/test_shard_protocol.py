"""The sharded decode's rank protocol on the host (no GPU): speculative first records, the boundary
check once the previous rank's tail arrives, and the correction of a false start -- in turn in one
process and over three gloo ranks.  The record predicate is the oracle's restatement."""

import os
import socket
import struct
import sys
from pathlib import Path

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as td  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from cubam_b200.shard import ShardProtocol  # noqa: E402
from oracle import bam_oracle as O  # noqa: E402

ROOT = Path(__file__).resolve().parents[1]
N_REF = 2


def _record(i: int, aux: bytes = b"") -> bytes:
    """A valid BAM record: read r<i>, 10M at position 100 i on reference 0, 10 bases."""
    name = b"r%d\0" % i
    pos, n_cig, l_seq = 100 * i, 1, 10
    cigar = struct.pack("<I", (10 << 4) | 0)
    seq, qual = bytes(5), bytes([30] * l_seq)
    body = struct.pack("<iiBBHHHIiii", 0, pos, len(name), 60, O.reg2bin(pos, pos + 10), n_cig, 0, l_seq, -1, -1, 0)
    body += name + cigar + seq + qual + aux
    return struct.pack("<i", len(body)) + body


def _data():
    """30 records; record 10 carries a complete fake record inside an aux string (a false start)."""
    recs = [_record(i) for i in range(30)]
    fake = _record(99)
    recs[10] = _record(10, b"XZH" + fake + b"\0")
    data = b"".join(recs)
    starts = np.cumsum([0] + [len(r) for r in recs])[:-1]
    fake_at = int(starts[10]) + len(recs[10]) - len(fake) - 1
    assert O.is_record(data, len(data), fake_at, N_REF)
    return data, starts, fake_at


class HostShard(ShardProtocol):
    """The protocol's primitives on host bytes, with the oracle's predicate (``hops`` linked records)."""

    def __init__(self, data: bytes, rank: int, hops: int = 0):
        self.data, self.rank, self.n_data, self.hops = data, rank, len(data), hops
        self.prev = b""

    def _first_record(self, limit):
        d, n = self.data, len(self.data)
        for o in range(min(limit, n)):
            if not O.is_record(d, n, o, N_REF):
                continue
            q, ok = o + 4 + struct.unpack_from("<i", d, o)[0], True
            for _ in range(self.hops):
                if q + 4 > n:
                    break
                if not O.is_record(d, n, q, N_REF):
                    bq = struct.unpack_from("<I", d, q)[0]  # a plausible record running past the end
                    ok = 33 <= bq <= (1 << 22) and q + 4 + bq > n
                    break
                q += 4 + struct.unpack_from("<i", d, q)[0]
            if ok:
                return o
        return -1

    def _chain(self, start, stop, tail_len):
        comb = (self.prev if tail_len else b"") + self.data
        try:
            offs, tail = O.record_chain(comb[start:stop], N_REF)
        except ValueError:
            return np.empty(0, np.int64), start, False
        return offs + start, start + int(tail), True

    def _place_tail(self, prev):
        self.prev = bytes(prev)
        return len(self.prev)

    @staticmethod
    def _shift(offs, t):
        return offs + t

    @staticmethod
    def _cat(a, b):
        return np.concatenate([a, b])


def _run_in_turn(parts, hops):
    prev, got, held = b"", [], []
    pos = 0  # global position of the combined bytes of the rank
    for r, part in enumerate(parts):
        sh = HostShard(part, r, hops)
        sh.speculate()
        offs, tail, ok = sh.confirm(prev)
        comb = prev + part
        got.append(offs + (pos - len(prev)))
        held.append(ok)
        pos += len(part)
        prev = comb[tail:]
    return np.concatenate(got), held, prev


def test_false_start_is_found_and_corrected():
    data, starts, fake_at = _data()
    want, tail = O.record_chain(data, N_REF)
    assert tail == len(data) and np.array_equal(want, starts)
    cut1, cut2 = fake_at - 7, int(starts[20]) + 5  # rank 1 starts inside record 10, before the fake
    parts = [data[:cut1], data[cut1:cut2], data[cut2:]]
    got, held, rest = _run_in_turn(parts, hops=0)
    assert np.array_equal(got, want) and rest == b""
    assert held == [True, False, True]  # rank 1's speculation took the fake record, and was corrected
    for hops in (1, 2, 4):  # whatever the speculation takes, the records are the whole chain's
        got, held, rest = _run_in_turn(parts, hops)
        assert np.array_equal(got, want) and rest == b""


@pytest.mark.parametrize("world", [1, 2, 5, 9])
def test_any_cuts_give_the_whole_chain(world):
    data, starts, _ = _data()
    rng = np.random.default_rng(world)
    cuts = sorted(rng.choice(np.arange(1, len(data)), world - 1, replace=False).tolist())
    bounds = [0] + cuts + [len(data)]
    parts = [data[a:b] for a, b in zip(bounds, bounds[1:])]
    got, _, rest = _run_in_turn(parts, hops=1)
    assert np.array_equal(got, starts) and rest == b""


def _gloo_rank(rank, world, port, q):
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    from cubam_b200.shard import recv_tail, send_tail
    from test_shard_protocol import HostShard, _data

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    td.init_process_group("gloo", rank=rank, world_size=world)
    try:
        data, starts, fake_at = _data()
        bounds = [0, fake_at - 7, int(starts[20]) + 5, len(data)]
        part = data[bounds[rank] : bounds[rank + 1]]
        sh = HostShard(part, rank, hops=0)
        sh.speculate()  # before anything arrives from the previous rank
        prev = recv_tail(rank, device="cpu")
        offs, tail, ok = sh.confirm(bytes(prev.tolist()))
        comb = bytes(prev.tolist()) + part
        send_tail(torch.tensor(list(comb[tail:]), dtype=torch.uint8), rank, world)
        q.put((rank, (offs + bounds[rank] - len(prev)).tolist(), ok))
    finally:
        td.destroy_process_group()


def test_three_gloo_ranks_correct_a_false_start():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_rank, args=(r, 3, port, q)) for r in range(3)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = dict((r, (o, ok)) for r, o, ok in (q.get(timeout=10) for _ in range(3)))
    data, starts, _ = _data()
    assert sum((res[r][0] for r in range(3)), []) == starts.tolist()
    assert [res[r][1] for r in range(3)] == [True, False, True]
