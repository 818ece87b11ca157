"""Sharding one file across ranks, host logic (no GPU): member boundaries with the chain rule, and the
tail exchange between two gloo ranks."""

import os
import socket
import struct
import sys
import zlib
from pathlib import Path

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as td  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from cubam_b200 import shard  # noqa: E402
from golden_io import GOLDEN  # noqa: E402
from oracle import bam_oracle  # noqa: E402

ROOT = Path(__file__).resolve().parents[1]


#: the 28-byte BGZF end-of-file member (an empty member holding one fixed-Huffman final block)
EOF_MEMBER = bytes.fromhex("1f8b08040000000000ff0600424302001b0003000000000000000000")


def _member(payload: bytes, level: int = 0) -> bytes:
    c = zlib.compressobj(level, zlib.DEFLATED, -15)
    body = c.compress(payload) + c.flush()
    bsize = 18 + len(body) + 8 - 1
    head = b"\x1f\x8b\x08\x04" + b"\0" * 4 + b"\0\xff" + struct.pack("<H", 6) + b"BC" + struct.pack("<HH", 2, bsize)
    return head + body + struct.pack("<II", zlib.crc32(payload), len(payload))


@pytest.mark.parametrize("name", ["mixed_b700.bam", "pairs.bam", "text_b300.gz"])
def test_boundaries_are_member_starts(name):
    raw = (GOLDEN / name).read_bytes()
    offs = set(int(x) for x in bam_oracle.scan_members(raw, True)[0])
    for world in range(1, 9):
        b = shard.member_boundaries(raw, world)
        assert len(b) == world + 1 and b[0] == 0 and b[-1] == len(raw)
        assert b == sorted(b)
        assert all(x in offs or x == len(raw) for x in b[1:-1])


def test_headers_inside_payloads_are_not_boundaries():
    fake = b"\x1f\x8b\x08\x04" + b"\0" * 6 + struct.pack("<H", 6) + b"BC" + struct.pack("<HH", 2, 99)
    members = [_member(fake * 50 + bytes([i]) * 300) for i in range(40)]  # stored: the fakes stay visible
    raw = b"".join(members) + EOF_MEMBER
    starts, o = [], 0
    for m in members:
        starts.append(o)
        o += len(m)
    for world in range(2, 12):
        for x in shard.member_boundaries(raw, world)[1:-1]:
            assert x in starts or x == o, x


def _rank(rank, world, port, q):
    sys.path.insert(0, str(ROOT))
    from cubam_b200 import shard as S

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    td.init_process_group("gloo", rank=rank, world_size=world)
    try:
        got = S.recv_tail(rank, device="cpu")
        mine = torch.tensor(list(b"tail-of-%d" % rank) * (rank + 1), dtype=torch.uint8)
        S.send_tail(mine, rank, world)
        q.put((rank, bytes(got.tolist())))
    finally:
        td.destroy_process_group()


def test_tails_pass_from_rank_to_rank_over_gloo():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 3, port, q)) for r in range(3)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = dict(q.get(timeout=10) for _ in range(3))
    assert got == {0: b"", 1: b"tail-of-0", 2: b"tail-of-1" * 2}


def _big_header_bam(tmp_path, member_bytes=700, extra_refs=3000):
    """A golden BAM rewritten with ``extra_refs`` more references in its header, in small members: the
    header spans many BGZF members."""
    import gzip

    raw = gzip.decompress((GOLDEN / "mixed_b700.bam").read_bytes())
    l_text = struct.unpack_from("<i", raw, 4)[0]
    n_ref = struct.unpack_from("<i", raw, 8 + l_text)[0]
    o = 12 + l_text
    refs = []
    for _ in range(n_ref):
        ln = struct.unpack_from("<i", raw, o)[0]
        refs.append(raw[o : o + 8 + ln])
        o += 8 + ln
    records = raw[o:]
    extra = [struct.pack("<i", 12) + b"extra%06d\0" % i + struct.pack("<i", 1000 + i) for i in range(extra_refs)]
    text = raw[8 : 8 + l_text] + b"".join(b"@SQ\tSN:extra%06d\tLN:%d\n" % (i, 1000 + i) for i in range(extra_refs))
    head = b"BAM\1" + struct.pack("<i", len(text)) + text + struct.pack("<i", n_ref + extra_refs) + b"".join(refs + extra)
    blob = head + records
    members = [_member(blob[i : i + member_bytes], 6) for i in range(0, len(blob), member_bytes)]
    p = tmp_path / "bighead.bam"
    p.write_bytes(b"".join(members) + EOF_MEMBER)
    return p, len(head)


def test_no_shard_but_the_first_starts_inside_the_header(tmp_path):
    p, hsize = _big_header_bam(tmp_path)
    raw = p.read_bytes()
    first_ok = shard.records_start_member(raw, hsize)
    # the header's members: their ISIZE up to first_ok cover the header
    o, covered = 0, 0
    while o < first_ok:
        bs = struct.unpack_from("<H", raw, o + 16)[0] + 1
        covered += struct.unpack_from("<I", raw, o + bs - 4)[0]
        o += bs
    assert o == first_ok and covered >= hsize > covered - 700
    for world in (2, 3, 7, 40):
        b = shard.member_boundaries(raw, world, hsize)
        assert all(x >= first_ok for x in b[1:])
        assert b == shard.member_boundaries(p, world, hsize)  # from windows of the file: the same cuts
