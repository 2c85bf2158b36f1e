"""The autotuner's shape cache: keyed by workload, saved and read back as JSON."""
from antiradiancecuts_b200 import api


def test_tuning_cache_round_trip(tmp_path):
    path = tmp_path / "autotune.json"
    c = api.TuningCache(str(path))
    assert c.get(api.TuningCache.key(1920, 1080, 1 << 20, 2, 0)) is None
    k = api.TuningCache.key(1920, 1080, 1 << 20, 2, 0)
    c.put(k, 11, [1.5, 2.25, 3.0])
    c.save()
    d = api.TuningCache(str(path))
    assert d.get(k) == 11 and d.entries[k]["times_ms"] == [1.5, 2.25, 3.0]
    assert d.get(api.TuningCache.key(1920, 1080, 1 << 20, 2, 3)) is None  # precision is part of the key
