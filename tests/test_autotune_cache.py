"""The autotuners' JSON cache (batch.cache_load / cache_store) on the CPU: a
missing, corrupt or non-object file reads as empty, entries merge, writes
leave no temporary file behind and an unwritable location is skipped."""
import json

from seiswave_taichi_b200 import batch as B


def test_cache_load_and_store(tmp_path, monkeypatch):
    p = tmp_path / "sub" / "autotune.json"
    monkeypatch.setenv("SEISWAVE_AUTOTUNE_CACHE", str(p))
    assert B.cache_load() == {}
    B.cache_store("a", 3)
    B.cache_store("b", 12)
    assert B.cache_load() == {"a": 3, "b": 12}
    assert json.loads(p.read_text()) == {"a": 3, "b": 12}
    assert [q.name for q in p.parent.iterdir()] == ["autotune.json"]
    p.write_text("{not json")
    assert B.cache_load() == {}
    p.write_text("[1, 2, 3]")
    assert B.cache_load() == {}
    B.cache_store("c", 1)  # a malformed file is replaced
    assert B.cache_load() == {"c": 1}


def test_cache_store_skips_an_unwritable_location(tmp_path, monkeypatch):
    blocker = tmp_path / "file"
    blocker.write_text("x")
    monkeypatch.setenv("SEISWAVE_AUTOTUNE_CACHE", str(blocker / "autotune.json"))
    B.cache_store("a", 1)  # its directory cannot be made: no error
    assert B.cache_load() == {}
