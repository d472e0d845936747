"""Autotuning cache (gromos_nb.tuning): keys, reuse without timing, atomic writes."""
import json

from gromos_nb import generators, tuning


def _sys(n=216, seed=3):
    return generators.spc_water_system(n, box=generators.box_for_waters(n), seed=seed, rcutp=0.8, rcutl=1.4)


def test_signature_depends_on_shape_not_coordinates():
    a, b = _sys(seed=3), _sys(seed=4)
    assert tuning.system_signature(a) == tuning.system_signature(b)
    c = _sys(n=343)
    assert tuning.system_signature(a) != tuning.system_signature(c)
    dev = {"name": "B200", "sms": 148}
    assert tuning.cache_key(dev, [tuning.system_signature(a)]) != tuning.cache_key({"name": "B200", "sms": 132},
                                                                                   [tuning.system_signature(a)])


def test_cached_choice_is_applied_without_timing(tmp_path):
    cache = tuning.TuningCache(str(tmp_path / "tune.json"))
    calls, applied = [], []

    def tune():
        calls.append(1)
        return {"water_layout": 2, "cluster_size": 8, "candidates": [{"water_layout": 2, "cluster_size": 8,
                                                                      "ms_per_step": 0.1}]}

    key = tuning.cache_key({"name": "B200", "sms": 148}, [tuning.system_signature(_sys())])
    r1 = tuning.tune_cached(cache, key, tune, lambda l, w: applied.append((l, w)))
    assert r1["cached"] is False and len(calls) == 1 and applied == []
    r2 = tuning.tune_cached(cache, key, tune, lambda l, w: applied.append((l, w)))
    assert r2["cached"] is True and len(calls) == 1 and applied == [(2, 8)]
    assert json.load(open(cache.path))[key]["cluster_size"] == 8


def test_unreadable_cache_reads_as_empty_and_is_rewritten(tmp_path):
    p = tmp_path / "tune.json"
    p.write_text("{not json")
    cache = tuning.TuningCache(str(p))
    assert cache.load() == {}
    cache.put("k", {"water_layout": 1, "cluster_size": 4})
    assert cache.get("k") == {"water_layout": 1, "cluster_size": 4}
    assert [f.name for f in tmp_path.iterdir()] == ["tune.json"]  # no temporary file left behind
