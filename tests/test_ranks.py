"""The multi-GPU timing rules of bench.py on two gloo ranks (CPU): every rank gets the slowest rank's
time, and the whole-job rate is the units of all ranks over it."""

import os
import socket
import sys
from pathlib import Path

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as td  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    sys.path.insert(0, str(ROOT))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    td.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.max_over_ranks(10.0 + 5.0 * rank)
        q.put((rank, ms, bench.whole_job(1e9, ms, world)))
    finally:
        td.destroy_process_group()


def test_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert [g[1] for g in got] == [15.0, 15.0]
    assert all(abs(g[2] - 2e9 / 0.015) < 1 for g in got)


def test_single_process_is_unchanged():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks(7.5) == 7.5
    assert bench.whole_job(3e9, 1000.0, 1) == 3e9
