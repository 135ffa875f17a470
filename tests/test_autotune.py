"""The autotuner's host logic on CPU: the cache key's step-count class, the candidate tiles and
the finalist round (timed by a fake runner, no GPU)."""
import pytest

from fast_shepherd_score_b200 import autotune


def test_steps_class_separates_short_and_long_launches():
    assert autotune.steps_class(1) == 0
    assert autotune.steps_class(3) == autotune.steps_class(16) == 1
    assert autotune.steps_class(17) == autotune.steps_class(200) == 2


def test_candidates_respect_the_mode_rules():
    esp = autotune.candidates("esp", 400, 50)
    assert esp and all(c["lanes_per_pose"] >= 4 for c in esp)         # large clouds
    assert {c["kernel_variant"] for c in esp} == {1, 2, 3, 4}           # no 8-point tile
    assert not any(c.get("accumulate") for c in esp)                    # tensor cores opt-in
    small = autotune.candidates("shape", 40, 50)
    assert 5 in {c["kernel_variant"] for c in small}
    assert {1, 2} <= {c["lanes_per_pose"] for c in small}
    pharm = autotune.candidates("pharm", 20, 50)
    assert {c["kernel_variant"] for c in pharm} == {0}
    assert max(c["lanes_per_pose"] for c in pharm) <= 8
    tc = autotune.candidates("esp", 400, 50, tensor_cores=True)
    assert {c.get("accumulate", 0) for c in tc} == {0, 2, 3}


def test_tune_keeps_the_fastest_finalist(monkeypatch, tmp_path):
    monkeypatch.setenv("FSS_AUTOTUNE_CACHE", str(tmp_path / "cache.json"))
    monkeypatch.setattr(autotune, "_MEM", {})
    monkeypatch.setattr(autotune, "_LOADED", True)
    cost = {1: 3.0, 2: 1.0, 3: 2.0, 4: 5.0, 5: 4.0}
    calls = []

    def fake_time(run, c, repeats):
        calls.append(c["kernel_variant"])
        return [cost[c["kernel_variant"]]] * repeats

    monkeypatch.setattr(autotune, "_time", fake_time)
    cands = [{"lanes_per_pose": 8, "chunks": 0, "cta_per_sm": 0, "kernel_variant": v}
             for v in cost]
    rec = autotune.tune(lambda **t: None, "key", cands, repeats=2, finalists=3,
                        final_repeats=2)
    assert rec["kernel_variant"] == 2 and rec["ms"] == pytest.approx(1.0)
    # the three fastest are re-timed in turns; the two slowest are not
    assert calls.count(4) == 1 and calls.count(5) == 1 and calls.count(2) == 3
    assert autotune.lookup("key")["kernel_variant"] == 2
