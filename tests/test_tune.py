"""Tuning cache and parameter application (host side; no kernel runs)."""

import json

import pytest

from cubam_b200 import _lib, tune


@pytest.fixture
def restore_params():
    yield
    for key, _ in tune.CANDIDATES.values():
        _lib.lib.cb_set_param(key, -1)


def test_apply_and_current(restore_params):
    tune.apply({"decode_root": 8, "copy_warps": 24, "chain_tile": 16384})
    cur = tune.current()
    assert cur["decode_root"] == 8 and cur["copy_warps"] == 24 and cur["chain_tile"] == 16384
    with pytest.raises(ValueError, match="copy_warps"):
        tune.apply({"copy_warps": 5})


def test_every_candidate_is_accepted(restore_params):
    for name, (_, values) in tune.CANDIDATES.items():
        for v in values:
            tune.apply({name: v})
            assert tune.current()[name] == v


def test_cache_round_trip(tmp_path, monkeypatch, restore_params):
    path = tmp_path / "sub" / "tune.json"
    monkeypatch.setattr(tune, "shape_key", lambda n, t: f"dev|members~{n}|isize~{t // max(n, 1)}")
    assert tune.apply_cached(1024, 1 << 26, path) is None
    params = dict(tune.current(), decode_root=6, inflate_form=3)
    tune.save_cache({tune.shape_key(1024, 1 << 26): {"params": params}}, path)
    assert json.loads(path.read_text())
    got = tune.apply_cached(1024, 1 << 26, path)
    assert got == params and tune.current()["decode_root"] == 6
    monkeypatch.setenv("CUBAM_B200_TUNE_CACHE", str(path))
    assert tune.cache_path() == path


def test_unreadable_cache_is_empty(tmp_path):
    p = tmp_path / "tune.json"
    p.write_text("{not json")
    assert tune.load_cache(p) == {}
    assert tune.load_cache(tmp_path / "missing.json") == {}


def test_pow2_rounding():
    assert tune._pow2(1) == 1 and tune._pow2(0) == 1
    assert tune._pow2(60000) == 65536 and tune._pow2(40000) == 32768


def test_nvtx_stage_ranges(monkeypatch):
    """Stage boundaries open and close one NVTX range per stage when tracing is on, none when off."""
    from cubam_b200 import _trace

    calls = []

    class FakeNvtx:
        def range_push(self, name):
            calls.append(("push", name))

        def range_pop(self):
            calls.append(("pop",))

    monkeypatch.setattr(_trace, "_nvtx", lambda: FakeNvtx())
    marked = []

    class Events:
        def mark(self, name):
            marked.append(name)

    for name in ("start", "scanned", "inflated", "chained", "decoded"):
        _trace.mark(Events(), name, enabled=True)
    assert marked == ["start", "scanned", "inflated", "chained", "decoded"]
    assert [c[0] for c in calls] == ["push", "pop", "push", "pop", "push", "pop", "push", "pop"]
    assert [c[1] for c in calls if c[0] == "push"] == ["cubam: member scan", "cubam: inflate", "cubam: record chain",
                                                       "cubam: record pass"]
    calls.clear()
    _trace.mark(None, "start", enabled=False)
    assert calls == []
