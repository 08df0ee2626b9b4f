"""Autotuner cache logic (CPU): keys, JSON round trip, the choice among timed candidates."""
import json

import pytest

from overlappingbls_b200 import tune


def test_keys():
    assert tune.step_key(96, 96, 65, "mixed") == "96x96x65:mixed"
    k1 = tune.ensemble_key([(96, 96, 65), (192, 192, 129), (96, 96, 65)], "mixed")
    k2 = tune.ensemble_key([(192, 192, 129), (96, 96, 65), (96, 96, 65)], "mixed")
    assert k1 == k2 == "192x192x129*1;96x96x65*2:mixed"


def test_cache_round_trip(tmp_path):
    p = str(tmp_path / "t.json")
    c = tune.load_cache(p)
    assert c == {"version": tune.CACHE_VERSION, "devices": {}}
    tune._entry(c, "dev", "step")["64x64x65:f64"] = {"params": {"fused": 0}, "ms": 1.0}
    tune.save_cache(c, p)
    assert tune.load_cache(p)["devices"]["dev"]["step"]["64x64x65:f64"]["params"] == {"fused": 0}
    with open(p, "w") as f:          # a cache of another version is ignored
        json.dump({"version": -1, "devices": {"x": 1}}, f)
    assert tune.load_cache(p)["devices"] == {}


def test_cache_path_env(monkeypatch, tmp_path):
    monkeypatch.setenv("OBL_TUNE_CACHE", str(tmp_path / "e.json"))
    assert tune.cache_path() == str(tmp_path / "e.json")
    assert tune.cache_path("x.json") == "x.json"


def test_pick():
    best, ms = tune.pick([({"a": 1}, 3.0), ({"a": 2}, None), ({"a": 3}, 2.0), ({"a": 4}, float("nan"))])
    assert best == {"a": 3} and ms == 2.0
    with pytest.raises(RuntimeError):
        tune.pick([({"a": 1}, None)])


def test_candidates():
    assert {"fused": 1, "fwd_cluster_size": 8, "fwd_clusters": 0} in tune.step_candidates(96, 96)
    assert all(c["fused"] != 1 for c in tune.step_candidates(96, 64))
    modes = {c["mode"] for c in tune.ENSEMBLE_CANDIDATES}
    assert modes == {"sequential", "concurrent", "persistent", "persistent_split"}
