"""cubam's kernel launcher through the ``cubam`` compatibility package, on the GPU: launches by
cubam's kernel names and argument lists give what this library's own API gives."""

import numpy as np
import pytest

from golden_io import GOLDEN

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

import cubam_b200  # noqa: E402
from cubam_b200 import compat  # noqa: E402
from cubam_b200.bam import _SIGNED_VIEW, _TYPES, FIELDS  # noqa: E402


def _same(a, b) -> bool:
    s = _SIGNED_VIEW.get(a.dtype)
    return a.dtype == b.dtype and (torch.equal(a, b) if s is None else torch.equal(a.view(s), b.view(s)))


@pytest.fixture(scope="module")
def k():
    compat.uninstall()
    compat.install()
    import cubam._kernels

    yield cubam._kernels
    compat.uninstall()


@pytest.fixture(scope="module")
def batch():
    return next(iter(cubam_b200.read_bam(GOLDEN / "mixed_b700.bam")))


def test_decode_fixed_by_name(k, batch):
    n = len(batch)
    cols = {f: torch.empty(n, dtype=_TYPES[f], device="cuda") for f in FIELDS}
    k.launch("decode_fixed", n, batch.data, batch.offset, np.int64(n), *(cols[f] for f in FIELDS))
    for f in FIELDS:
        assert _same(cols[f], batch.columns[f]), f


def test_find_tag_and_hashes_by_name(k, batch):
    n = len(batch)
    tag = batch.tag("CB")
    t = torch.empty(n, dtype=torch.uint8, device="cuda")
    voff = torch.empty(n, dtype=torch.int64, device="cuda")
    vlen = torch.empty(n, dtype=torch.int32, device="cuda")
    ival = torch.empty(n, dtype=torch.int64, device="cuda")
    k.launch("find_tag", n, batch.data, batch.offset, np.int64(n), np.uint8(ord("C")), np.uint8(ord("B")),
             t, voff, vlen, ival)
    assert torch.equal(t, tag.type) and torch.equal(voff, tag.offset) and torch.equal(vlen, tag.length)
    h = torch.empty(n, dtype=torch.uint64, device="cuda")
    k.kernel("name_hash")((n // 256 + 1,), (256,), (batch.data, batch.offset, np.int64(n), h))
    assert _same(h, batch.name_hash())


def test_copy_spans(k, batch):
    sizes = batch.record_sizes()
    dst_off = torch.cumsum(sizes, 0) - sizes
    out = torch.zeros(int(sizes.sum()), dtype=torch.uint8, device="cuda")
    k.copy_spans(batch.data, out, batch.offset.cpu().numpy(), dst_off, sizes)
    start, end = int(batch.offset[0]), int(batch.offset[-1] + sizes[-1])
    assert torch.equal(out, batch.data[start:end])
