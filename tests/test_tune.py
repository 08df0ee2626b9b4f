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
    assert modes == {"sequential", "concurrent", "persistent", "persistent_split", "persistent_flow"}


def test_step_candidates_include_solve_schedules():
    c = tune.step_candidates(512, 512)
    assert {"fused": 0, "tdma_reg": 0, "tdma_segments": 0} in c
    assert {"fused": 0, "tdma_reg": 1, "tdma_segments": 16} in c


def test_build_sweep_caches_the_fastest_schedule(tmp_path, monkeypatch):
    """tune_build times every built variant (here a fake timer keyed by library path),
    caches every timing and the fastest schedule, and tuned_defines returns its -D list."""
    out = str(tmp_path / "variants")
    names = ["default", "cols_4w4l", "rows_pad16"]
    import os
    os.makedirs(out)
    for n in names[1:]:
        open(tune.variant_path(out, n), "w").close()
    fake = {None: 5.3, tune.variant_path(out, "cols_4w4l"): 5.9, tune.variant_path(out, "rows_pad16"): 5.1}
    monkeypatch.setattr(tune, "bench_ms", lambda lib, *a, **k: fake[lib])
    cache = str(tmp_path / "t.json")
    name, defines, ms = tune.tune_build("512x512x256", out, names, path=cache, device="B200")
    assert name == "rows_pad16" and defines == ["OBL_SIDX_SHIFT=4"] and ms == 5.1
    ent = tune.load_cache(cache)["devices"]["B200"]["build"]["512x512x256"]
    assert len(ent["timings"]) == 3
    assert tune.tuned_defines("512x512x256", path=cache) == ["OBL_SIDX_SHIFT=4"]
    assert tune.tuned_defines("64x64x64", path=cache) == []


def test_build_candidates_are_definitions():
    for name, defs in tune.BUILD_CANDIDATES.items():
        assert all("=" in d and d.startswith("OBL_") for d in defs), name
    assert tune.BUILD_CANDIDATES["default"] == []


def test_build_sweep_in_parts_merges(tmp_path, monkeypatch):
    out = str(tmp_path / "v")
    import os
    os.makedirs(out)
    for n in ("cols_4w4l", "rows_pad16"):
        open(tune.variant_path(out, n), "w").close()
    fake = {None: 5.3, tune.variant_path(out, "cols_4w4l"): 5.0, tune.variant_path(out, "rows_pad16"): 5.6}
    monkeypatch.setattr(tune, "bench_ms", lambda lib, *a, **k: fake[lib])
    cache = str(tmp_path / "t.json")
    tune.tune_build("w", out, ["default", "cols_4w4l"], path=cache, device="d")
    name, _, ms = tune.tune_build("w", out, ["default", "rows_pad16"], path=cache, device="d")
    ent = tune.load_cache(cache)["devices"]["d"]["build"]["w"]
    assert sorted(p["name"] for p, _ in ent["timings"]) == ["cols_4w4l", "default", "rows_pad16"]
    assert name == "cols_4w4l" and ms == 5.0
