"""The autotune cache: a choice recorded for a workload shape is applied to a later context of the same
shape that has no launch of its own, and to nothing else."""

import json

import pytest

from exmarg_b200 import pe


class FakeContext:
    def __init__(self, nm=2048, n_time=32768, store_shape=(53, 87, 49, 200, 219, 0), total=183 << 30):
        self.nm, self.n_time, self.store_shape, self.device_total = nm, n_time, store_shape, total
        self.gather_cfg = None
        self.gather_chunk_pct = 100
        self.calls = []

    def set_gather_cfg(self, cfg, chunk_pct=0):
        self.calls.append((cfg, chunk_pct))
        self.gather_cfg = cfg


@pytest.fixture
def cache(tmp_path, monkeypatch):
    path = tmp_path / "sub" / "autotune.json"
    monkeypatch.setenv("EXMARG_B200_TUNE_CACHE", str(path))
    return path


def test_record_then_apply(cache):
    a = FakeContext()
    pe.record_tuned(a, 1024, 1024, 2, 200, [97.0, 98.0, 99.0])
    assert json.loads(cache.read_text())[pe.tune_key(a, 1024, 1024)]["shape"] == 2
    b = FakeContext()
    e = pe.apply_tuned(b, 1024, 1024)
    assert e["chunk_pct"] == 200 and b.calls == [(2, 200)]


def test_other_shapes_and_own_choices_are_left_alone(cache):
    pe.record_tuned(FakeContext(), 1024, 1024, 2, 200)
    for ctx, walk in ((FakeContext(nm=1024), 1024), (FakeContext(n_time=16384), 1024), (FakeContext(), 512),
                      (FakeContext(total=80 << 30), 1024)):
        assert pe.apply_tuned(ctx, walk, walk) is None and ctx.calls == []
    own = FakeContext()
    own.gather_cfg = 0
    assert pe.apply_tuned(own, 1024, 1024) is None and own.calls == []
    child = FakeContext()
    child.parent = object()
    assert pe.apply_tuned(child, 1024, 1024) is None and child.calls == []


def test_unreadable_cache_is_ignored(cache):
    cache.parent.mkdir(parents=True)
    cache.write_text("{not json")
    assert pe.apply_tuned(FakeContext(), 1024, 1024) is None
    pe.record_tuned(FakeContext(), 1024, 1024, 1, 150)     # rewritten whole
    assert pe.apply_tuned(FakeContext(), 1024, 1024)["shape"] == 1
