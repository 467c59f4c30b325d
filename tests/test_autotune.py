"""Autotuner of the windowed tiling: workload keys, the JSON cache, candidate
selection and its bit-for-bit agreement check (CPU; a fake runner stands in
for the device timing).  The device run is in test_gpu_autotune.py."""
from __future__ import annotations

import json

import numpy as np
import pytest

from summit_b200 import autotune


class FakeSession:
    N = 5000


def _ws():
    return np.array([0, 300, 1700, 2000, 5000], dtype=np.int64)


def test_workload_key_is_stable_and_shape_sensitive():
    k1 = autotune.workload_key("B200", 5000, 20000, 24, 50, _ws())
    assert k1 == autotune.workload_key("B200", 5000, 20000, 24, 50, _ws().copy())
    assert k1 != autotune.workload_key("B200", 5000, 20000, 24, 10, _ws())
    assert k1 != autotune.workload_key("H100", 5000, 20000, 24, 50, _ws())
    assert k1 != autotune.workload_key("B200", 5000, 20000, 24, 50, np.array([0, 5000]))


def test_select_picks_fastest_and_checks_scores():
    ld = np.arange(12.0).reshape(6, 2)
    times = {4: 3.0, 8: 2.0, 16: 2.5}
    rec = autotune.select([{"p1_sb_per_cta": s, "batch_gb": 8.0} for s in times],
                          lambda c: (times[c["p1_sb_per_cta"]], ld))
    assert rec["config"]["p1_sb_per_cta"] == 8 and rec["ms"] == 2.0
    assert len(rec["trials"]) == 3
    bad = iter([ld, ld + 1e-12])
    with pytest.raises(RuntimeError):
        autotune.select([{"p1_sb_per_cta": 4}, {"p1_sb_per_cta": 8}], lambda c: (1.0, next(bad)))
    with pytest.raises(ValueError):
        autotune.select([], lambda c: (1.0, ld))


def test_tune_uses_and_refreshes_the_cache(tmp_path):
    path = tmp_path / "tune.json"
    calls = []

    def run(c):
        calls.append(c)
        return 10.0 / c["p1_sb_per_cta"], np.ones(3)

    annot = np.ones((5000, 2))
    cands = [{"p1_sb_per_cta": s, "batch_gb": 8.0} for s in (4, 16)]
    r1 = autotune.tune_windowed(FakeSession(), annot, _ws(), 50, 1000, 1, candidates=cands,
                                cache=autotune.TuneCache(path), run=run)
    assert not r1["cached"] and r1["config"]["p1_sb_per_cta"] == 16 and len(calls) == 2
    stored = json.loads(path.read_text())
    assert r1["key"] in stored and stored[r1["key"]]["config"]["p1_sb_per_cta"] == 16
    r2 = autotune.tune_windowed(FakeSession(), annot, _ws(), 50, 1000, 1, candidates=cands,
                                cache=autotune.TuneCache(path), run=run)
    assert r2["cached"] and len(calls) == 2
    r3 = autotune.tune_windowed(FakeSession(), annot, _ws(), 50, 1000, 1, candidates=cands,
                                cache=autotune.TuneCache(path), run=run, force=True)
    assert not r3["cached"] and len(calls) == 4


def test_cache_survives_a_corrupt_file(tmp_path):
    path = tmp_path / "tune.json"
    path.write_text("{not json")
    c = autotune.TuneCache(path)
    assert c.get("x") is None
    c.put("x", {"config": autotune.DEFAULT_CONFIG, "ms": 1.0})
    c.save()
    assert autotune.TuneCache(path).get("x")["ms"] == 1.0


def test_default_candidates_cover_the_knobs():
    cands = autotune.default_candidates()
    assert {c["batch_gb"] for c in cands} == {4.0, 8.0, 16.0}
    assert len({c["p1_sb_per_cta"] for c in cands}) >= 3
    assert all(set(c) == set(autotune.DEFAULT_CONFIG) for c in cands)
    assert {c["p2_bins"] for c in cands} == {0, 1}
