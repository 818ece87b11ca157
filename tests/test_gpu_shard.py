"""One file decoded as N shards (run in turn on one GPU, tails handed on): the concatenated records,
columns and tags equal the whole-file decode, whatever N."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from cubam_b200 import batch, shard, synth  # noqa: E402
from cubam_b200.bam import BamHeader  # noqa: E402
from cubam_b200.synth import Config  # noqa: E402
from golden_io import GOLDEN  # noqa: E402

TAGS = ("CB", "UB", "GN")
FIELDS = ("ref", "pos", "end", "mapq", "flag", "nref", "npos", "tlen", "l_seq", "clip_left", "clip_right")


@pytest.fixture(scope="module")
def paths(tmp_path_factory):
    d = tmp_path_factory.mktemp("shard")
    p = d / "g.bam"
    synth.write_bam(p, Config("g", 1, 60_000, 61, level=-1, stored_frac=0.03))
    return [p, GOLDEN / "pairs.bam", GOLDEN / "mixed_b700.bam"]


@pytest.mark.parametrize("world", [1, 2, 3, 7])
def test_shards_equal_the_whole_file(paths, world):
    for path in paths:
        header = BamHeader.read(path)
        whole = batch.decode_many([(batch.load_compressed(path), header)], tags=TAGS)[0]
        parts = shard.decode_shards_in_turn(path, world, tags=TAGS)
        assert sum(len(p) for p in parts) == len(whole)
        # each part's bytes start where the previous part's complete records end
        pos, offs = 0, []
        for p in parts:
            offs.append(p.offset.cpu().numpy() + pos)
            pos += (int(p.offset[-1].item()) + _size(p, -1)) if len(p) else 0
        assert np.array_equal(np.concatenate(offs), whole.offset.cpu().numpy())
        for k in FIELDS:
            got = torch.cat([p.columns[k] for p in parts])
            assert torch.equal(got, whole.columns[k]), k
        for t in TAGS:
            for x in ("type", "length", "value"):
                got = torch.cat([getattr(p.tags[t], x) for p in parts if len(p)])
                assert torch.equal(got, getattr(whole.tags[t], x)), (t, x)


def _size(p, i):
    o = int(p.offset[i].item())
    return 4 + int.from_bytes(p.data[o : o + 4].cpu().numpy().tobytes(), "little")


def test_shards_with_a_header_of_many_members(tmp_path):
    """A header spread over ~150 BGZF members (3,000 extra references) and 7 ranks: no rank but the
    first starts inside it, and the shards give the whole file's records."""
    from test_shard_host import _big_header_bam

    p, _ = _big_header_bam(tmp_path)
    header = BamHeader.read(p)
    whole = batch.decode_many([(batch.load_compressed(p), header)], tags=TAGS)[0]
    for world in (2, 7):
        parts = shard.decode_shards_in_turn(p, world, tags=TAGS)
        assert sum(len(x) for x in parts) == len(whole)
        for k in FIELDS:
            got = torch.cat([x.columns[k] for x in parts])
            assert torch.equal(got, whole.columns[k]), k
