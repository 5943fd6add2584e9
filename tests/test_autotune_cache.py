"""The autotuner's cache (CPU): tuned values are stored per device under
$XDG_CACHE_HOME and read back by a fresh process state, including the
checkpoint interval k of gauge runs and the per-arithmetic tile heights."""
import json

from diffswe2d_b200 import autotune


def test_cache_round_trip(tmp_path, monkeypatch):
    monkeypatch.setenv("XDG_CACHE_HOME", str(tmp_path))
    monkeypatch.setattr(autotune, "_device_key", lambda device: "TestGPU/148")
    monkeypatch.setattr(autotune, "_tuned", {})
    entry = autotune._load("cuda")
    assert entry == {}
    entry["rows"] = [8, 16, 32, 8]
    entry["rows_fast"] = [16, 16, 32, 16]
    entry["checkpoint_every"] = {
        "exact/4x244x393/1125x0.02/6g/auto": {"k": 64, "timing_ms": {"32": 9.0, "64": 7.5},
                                               "intervals_timed": 300}}
    autotune._store("cuda", entry)
    on_disk = json.loads((tmp_path / "diffswe2d_b200" / "autotune.json").read_text())
    assert on_disk["TestGPU/148"]["checkpoint_every"]["exact/4x244x393/1125x0.02/6g/auto"]["k"] == 64
    monkeypatch.setattr(autotune, "_tuned", {})  # a new process
    assert autotune.tuned_rows(5000, "cuda") == 8
    assert autotune.tuned_rows(5000, "cuda", "fast") == 16
    assert autotune.tuned_rows(1 << 24, "cuda", "fast") == 16
    got = autotune.checkpoint_tuning("cuda", "exact/4x244x393")
    assert list(got.values())[0]["k"] == 64


def test_defaults_without_cache(tmp_path, monkeypatch):
    monkeypatch.setenv("XDG_CACHE_HOME", str(tmp_path))
    monkeypatch.setattr(autotune, "_device_key", lambda device: "Other/1")
    monkeypatch.setattr(autotune, "_tuned", {})
    assert autotune.tuned_rows(100, "cuda") == autotune.DEFAULT_ROWS[0]
    assert autotune.tuned_ensemble_rows("cuda", "fast") == 16
    assert autotune.checkpoint_tuning("cuda") == {}
