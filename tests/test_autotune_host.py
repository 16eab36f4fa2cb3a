"""Autotuner cache (voxelmapping_b200.autotune) on the host: entries are
stored and found by key, the user cache wins over the shipped table, and a
missing or corrupt cache falls back cleanly."""
import json

from voxelmapping_b200 import autotune as AT


def test_store_and_lookup(tmp_path, monkeypatch):
    cache = tmp_path / "t.json"
    monkeypatch.setenv("VMAP_TUNING_CACHE", str(cache))
    monkeypatch.setattr(AT, "SHIPPED", tmp_path / "shipped.json")
    k = AT.key_for("map", "f32", 640, 480)
    assert AT.lookup(k) == (None, None)
    (tmp_path / "shipped.json").write_text(json.dumps({k: {"config": {"fuse_ctas_per_sm": 8}}}))
    cfg, src = AT.lookup(k)
    assert src == "shipped" and cfg["fuse_ctas_per_sm"] == 8 and cfg["alloc_ctas_per_sm"] == 0
    AT.store(k, {f: 3 for f in AT.FIELDS}, {"note": "x"})
    cfg, src = AT.lookup(k)
    assert src == "cache" and all(cfg[f] == 3 for f in AT.FIELDS)
    kb = AT.key_for("batch", "f16", 640, 480, 32)
    assert kb != k and "maps=32" in kb
    AT.store(kb, {"raycast_ctas_per_sm": 2})
    assert AT.lookup(kb)[0]["raycast_ctas_per_sm"] == 2 and AT.lookup(k)[1] == "cache"
    cache.write_text("{not json")
    assert AT.lookup(k)[1] == "shipped"


def test_candidates_are_valid_launch_values():
    for f in AT.FIELDS:
        if f.endswith("_ctas_per_sm"):  # grids: 0 (default) .. 64 CTAs per SM
            assert all(0 <= c <= 64 for c in AT.CANDIDATES[f]), f
    assert set(AT.CANDIDATES["raycast_tile_order"]) == {0, 1, 2}
    assert set(AT.STAGE) | {"mesh_ctas_per_sm", "batch_schedule"} | set(AT.RAYCAST_PARAMS) == set(AT.FIELDS)
    assert set(AT.CANDIDATES["batch_schedule"]) == {1, 2}
    assert set(AT.CANDIDATES["raycast_tile_width"]) == {4, 8, 16}
    assert set(AT.CANDIDATES["raycast_threads_per_cta"]) == {128, 256}
