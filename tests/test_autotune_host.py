"""Host logic of the half-step autotuner (no GPU): the cache key's size classes, the choice of the fastest candidate,
the cache round trip and `force`.  The backend is replaced by a stand-in whose half-step times depend on the
tuning word, so only the tuner's own bookkeeping is under test."""
import json

import pytest

from cumulus3d_b200 import autotune, scenes


class _FakeSession:
    def __init__(self, tuning, log):
        self.tuning, self.log = tuning, log

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False

    def run_resident(self, views, p):
        self.log.append((self.tuning, tuple(views), p.iterations))

    def synchronize(self):
        pass

    def set_profiling(self, on):
        pass

    def reset_stats(self):
        pass

    def kernel_stats(self, kind):
        return {"ms": {0: 5.0, 2: 4.0, 3: 3.5, 4: 2.5, 6: 3.0, 7: 2.75, 8: 2.6, 10: 2.7, 16: 2.9, 18: 2.8, 42: 2.65,
                       90: 2.85}[self.tuning]}


class _FakeBackend:
    log = []

    def __init__(self, device=0, math="parity", tuning=0):
        self.tuning = tuning

    def name(self):
        return "Fake B200"

    def close(self):
        pass

    def begin(self, inp):
        return _FakeSession(self.tuning, _FakeBackend.log)


@pytest.fixture
def fake(monkeypatch):
    _FakeBackend.log = []
    monkeypatch.setattr(autotune, "PatchMatchBackend", _FakeBackend)
    return _FakeBackend


def test_key_size_classes():
    small = scenes.workload_small(96, 72).input
    assert autotune._key("G", small, "parity") == "G|r3|s1|parity|S|n2"
    c1 = scenes.workload_c1().input
    assert autotune._key("G", c1, "fast").endswith("|r5|s1|fast|S|n2")  # 0.31 Mpix, 2 sources


def test_key_of_a_mixed_batch_names_every_size_class_and_the_source_count():
    """A batch of several image sizes keys on all of its size classes (not on its first view's) and on its largest
    source count; the tuner's views include one of every size class."""
    inp = scenes.workload_small(96, 72, views=4).input
    big = scenes.workload_small(1024, 768, views=2).input
    inp.views = inp.views + big.views
    inp.views[-1].sources = list(range(5))
    assert autotune._key("G", inp, "parity") == "G|r3|s1|parity|MS|n5"


def test_tuning_views_cover_every_size_class(fake, tmp_path):
    inp = scenes.workload_small(96, 72, views=6).input
    n = len(inp.views)
    big = scenes.workload_small(1024, 768, views=1).input
    inp.views = inp.views + big.views
    autotune.tune(inp, cache=tmp_path / "t.json", max_views=2, candidates=(0,))
    assert fake.log[0][1] == (0, n)


def test_picks_fastest_and_caches(fake, tmp_path):
    inp = scenes.workload_small(96, 72, views=6, positions=2).input
    cache = tmp_path / "tune.json"
    r = autotune.tune(inp, cache=cache, max_views=4)
    assert r["tuning"] == 4 and not r["cached"]
    assert set(r["ms"]) == {str(t) for t in autotune.CANDIDATES}
    # every candidate ran a converging warm-up of two iterations, then a timed iteration, on the first 4 views
    assert sorted({t for t, _, _ in fake.log}) == sorted(autotune.CANDIDATES)
    assert all(v == (0, 1, 2, 3) for _, v, _ in fake.log)
    assert [it for _, _, it in fake.log] == [2, 1] * len(autotune.CANDIDATES)
    assert len(fake.log) == 2 * len(autotune.CANDIDATES)
    stored = json.loads(cache.read_text())
    assert stored[r["key"]]["tuning"] == 4
    fake.log.clear()
    again = autotune.tune(inp, cache=cache)
    assert again["cached"] and again["tuning"] == 4 and fake.log == []
    forced = autotune.tune(inp, cache=cache, force=True, candidates=(0, 6))
    assert forced["tuning"] == 6 and not forced["cached"]


def test_unreadable_cache_is_ignored(fake, tmp_path):
    inp = scenes.workload_small(96, 72).input
    cache = tmp_path / "tune.json"
    cache.write_text("{not json")
    assert autotune.tune(inp, cache=cache, candidates=(3, 7))["tuning"] == 7
