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


def test_calibration_chooses_the_fastest_value_within_the_target():
    from antiradiancecuts_b200 import learned

    values = (0.01, 0.05, 0.1)
    res = [[{"rel_rmse": 0.004}, {"rel_rmse": 0.006}],   # 0.01: within
           [{"rel_rmse": 0.008}, {"rel_rmse": 0.0094}],  # 0.05: within (worst scene 0.94%)
           [{"rel_rmse": 0.007}, {"rel_rmse": 0.012}]]   # 0.1: one scene over the target
    assert learned.choose(values, res, 0.0095) == 0.05
    assert learned.choose(values, res, 0.001) is None
    img = [[1.0, 2.0, 3.0], [0.5, 0.5, 0.5]]
    ref = [[1.0, 2.0, 3.0], [0.4, 0.5, 0.5]]
    e = learned.image_errors(img, ref, [[2.0, 2.0, 3.0], [0.6, 0.6, 0.6]], [[1.0, 0.0, 0.0], [0.2, 0.1, 0.1]])
    assert abs(e["max_rel_err"] - 0.1 / 0.8) < 1e-12 and e["rel_rmse"] > 0
