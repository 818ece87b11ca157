"""The member scan that allocates nothing gives what the member scan with a workspace gives.

``cb_scan_members_noalloc`` is for callers that cannot allocate device memory
for a workspace (a serving process whose device memory belongs to one pool, a
caller from another runtime with no device allocator, a loop that must not let
cudaMalloc synchronise the device): its scratch is a fixed array inside the
library, for inputs of at most 16 MiB.  Both entry points are called through
the C ABI on the same inputs; every call of the allocation-free one must give
the same job table and summary, byte for byte, two calls in a row (the shared
scratch keeps the previous call's contents).  This file is collected last on
purpose.
"""

import ctypes

import pytest

from golden_io import GOLDEN

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from cubam_b200 import _lib  # noqa: E402

MAX = 16 << 20
SUMMARY = ctypes.sizeof(_lib.ScanSummary)


def _device(raw: bytes) -> torch.Tensor:
    return torch.frombuffer(bytearray(raw), dtype=torch.uint8).cuda()


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def _with_workspace(buf: torch.Tensor, eof: bool, cap: int):
    n = int(buf.numel())
    ws = torch.empty(max(int(_lib.lib.cb_scan_workspace_bytes(n)), 256), dtype=torch.uint8, device="cuda")
    jobs = torch.zeros(cap * _lib.JOB_BYTES, dtype=torch.uint8, device="cuda")
    summ = torch.zeros(SUMMARY, dtype=torch.uint8, device="cuda")
    rc = _lib.lib.cb_scan_members(buf.data_ptr(), n, int(eof), 0, jobs.data_ptr(), cap, summ.data_ptr(),
                                  ws.data_ptr(), ws.numel(), _stream())
    assert rc == _lib.OK
    torch.cuda.synchronize()
    return jobs.cpu().numpy().tobytes(), summ.cpu().numpy().tobytes()


def _no_alloc(buf: torch.Tensor, eof: bool, cap: int):
    n = int(buf.numel())
    jobs = torch.zeros(cap * _lib.JOB_BYTES, dtype=torch.uint8, device="cuda")
    summ = torch.zeros(SUMMARY, dtype=torch.uint8, device="cuda")
    rc = _lib.lib.cb_scan_members_noalloc(buf.data_ptr(), n, int(eof), 0, jobs.data_ptr(), cap, summ.data_ptr(),
                                          _stream())
    assert rc == _lib.OK, _lib.lib.cb_last_error()
    torch.cuda.synchronize()
    return jobs.cpu().numpy().tobytes(), summ.cpu().numpy().tobytes()


CASES = [
    ("mixed_b700.bam", True),  # about 1,500 small members
    ("text_b300.gz", True),  # members of 300 bytes of data
    ("pairs.bam", True),
    ("mixed_b65280.bam", False),  # a chunk that ends inside a member: the carry case
]


def _input(name: str, eof: bool) -> bytes:
    raw = (GOLDEN / name).read_bytes()
    return raw if eof else raw[: len(raw) * 2 // 3]


@pytest.mark.parametrize(("name", "eof"), CASES)
def test_no_alloc_scan_matches_the_workspace_scan(name, eof):
    buf = _device(_input(name, eof))
    cap = int(buf.numel()) // 26 + 2
    want = _with_workspace(buf, eof, cap)
    status = _lib.ScanSummary.from_buffer_copy(want[1]).status
    assert status == _lib.OK
    for _ in range(2):
        assert _no_alloc(buf, eof, cap) == want


def test_no_alloc_scan_after_another_input():
    """The scratch holds the previous call's state; a call on other data must not see it."""
    big = _device(_input("mixed_b700.bam", True))
    small = _device(_input("pairs.bam", True))
    cap = int(big.numel()) // 26 + 2
    want_small = _with_workspace(small, True, cap)
    _no_alloc(big, True, cap)
    assert _no_alloc(small, True, cap) == want_small
    assert _no_alloc(small, True, cap) == want_small


def test_no_alloc_scan_rejects_inputs_beyond_its_scratch():
    buf = _device(b"\0" * 64)
    jobs = torch.zeros(_lib.JOB_BYTES, dtype=torch.uint8, device="cuda")
    summ = torch.zeros(SUMMARY, dtype=torch.uint8, device="cuda")
    rc = _lib.lib.cb_scan_members_noalloc(buf.data_ptr(), MAX + 1, 1, 0, jobs.data_ptr(), 1, summ.data_ptr(),
                                          _stream())
    assert rc == _lib.CAPACITY
    assert b"16 MiB" in _lib.lib.cb_last_error()
