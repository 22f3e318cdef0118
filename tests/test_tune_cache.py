"""The autotuner's on-disk cache (CPU: file handling only; the GPU tests of
test_autotune.py cover the measured choices themselves)."""

import json

from hit_solver_b200 import _lib, autotune


def test_disk_cache_round_trip(tmp_path, monkeypatch):
    path = tmp_path / "sub" / "tuning.json"
    monkeypatch.setenv("HITB200_TUNE_CACHE", str(path))
    assert autotune.cache_path() == path
    key = autotune._disk_key((1, ((512, 512, 1, 0, 4, 1, 1, 1, 5),)))
    assert autotune._disk_load(key) is None
    autotune._disk_store(key, [1, 0, 1, 0, 1, 0])
    assert autotune._disk_load(key) == [1, 0, 1, 0, 1, 0]
    # a second entry is merged, not overwriting the first
    key2 = autotune._disk_key((0, ((64, 48, 1, 0, 4, 1, 1, 1, 5),)))
    autotune._disk_store(key2, [0, 0, 0, 1, 0, 0])
    data = json.loads(path.read_text())
    assert data[key] == [1, 0, 1, 0, 1, 0] and data[key2] == [0, 0, 0, 1, 0, 0]
    assert not list(path.parent.glob("*.tmp"))


def test_disk_cache_rejects_bad_entries(tmp_path, monkeypatch):
    path = tmp_path / "tuning.json"
    monkeypatch.setenv("HITB200_TUNE_CACHE", str(path))
    key = autotune._disk_key(("x",))
    path.write_text(json.dumps({key: [2, 0, 0, 0, 0, 0]}))
    assert autotune._disk_load(key) is None
    path.write_text(json.dumps({key: [0] * (_lib.TUNE_COUNT + 1)}))
    assert autotune._disk_load(key) is None
    path.write_text("not json")
    assert autotune._disk_load(key) is None
    autotune._disk_store(key, [0, 1, 0, 0, 1, 1])  # a corrupt file is replaced
    assert autotune._disk_load(key) == [0, 1, 0, 0, 1, 1]


def test_disk_cache_off(tmp_path, monkeypatch):
    monkeypatch.setenv("HITB200_TUNE_CACHE", "off")
    assert autotune.cache_path() is None
    key = autotune._disk_key(("y",))
    autotune._disk_store(key, [1, 1, 1, 0, 0, 1])
    assert autotune._disk_load(key) is None


def test_lookup_fills_memory_cache_from_disk(tmp_path, monkeypatch):
    monkeypatch.setenv("HITB200_TUNE_CACHE", str(tmp_path / "t.json"))
    autotune.clear_cache()
    key = (1, ((96, 96, 0, 0, 4, 0, 0, 0, 1),))
    autotune._disk_store(autotune._disk_key(key), [1, 1, 0, 0, 1, 0])
    assert autotune._lookup(key, use_cache=False) is None
    assert autotune._lookup(key, use_cache=True) == [1, 1, 0, 0, 1, 0]
    assert autotune._cache[key] == [1, 1, 0, 0, 1, 0]
    autotune.clear_cache()
