"""The launch-shape autotuner's selection and cache logic, on the host (fake engine)."""
import json

from gip_b200 import autotune


class FakeEngine:
    """Times each grid size from a table, records the launches it was given."""

    def __init__(self, ms_by_blocks):
        self.ms = ms_by_blocks
        self.blocks = None
        self.timed = []

    def set_launch(self, blocks, threads):
        self.blocks = blocks

    def kernel_time(self, kernel, reps=15):
        self.timed.append(self.blocks)
        return self.ms[self.blocks], 0.0


def test_picks_fastest_grid_and_caches(tmp_path, monkeypatch):
    monkeypatch.setattr(autotune, "_sm_count", lambda: 148)
    monkeypatch.setattr(autotune, "_CACHE", {})
    ms = {148: 1.0, 296: 0.7, 592: 0.5, 888: 0.6, 1184: 0.9}
    E = FakeEngine(ms)
    path = str(tmp_path / "tune.json")
    r = autotune.tune(E, "mixed", rows=1000, nnz=7000, path=path)
    assert r["blocks"] == 592 and not r["cached"] and E.blocks == 592
    assert sorted(E.timed) == sorted(ms)
    assert json.load(open(path)) == {"mixed:1000:7000": 592}
    # the same operator class again: no timing, the cached grid applied
    F = FakeEngine(ms)
    r = autotune.tune(F, "mixed", rows=1000, nnz=7000, path=path)
    assert r == {"blocks": 592, "cached": True} and F.timed == [] and F.blocks == 592
    # a fresh process reads the file
    monkeypatch.setattr(autotune, "_CACHE", {})
    G = FakeEngine(ms)
    assert autotune.tune(G, "mixed", rows=1000, nnz=7000, path=path)["cached"]
    assert G.timed == [] and G.blocks == 592


def test_grid_capped_and_classes_separate(monkeypatch):
    monkeypatch.setattr(autotune, "_sm_count", lambda: 2000)
    monkeypatch.setattr(autotune, "_CACHE", {})
    E = FakeEngine({2000: 0.3, 4000: 0.2, 8192: 0.25})
    r = autotune.tune(E, "fp64", rows=5, nnz=9, multiples=(1, 2, 8, 16))
    assert max(E.timed) == 8192 and r["blocks"] == 4000
    E2 = FakeEngine({2000: 0.1, 4000: 0.2, 8192: 0.25})
    assert autotune.tune(E2, "fp64", rows=6, nnz=9, multiples=(1, 2, 8))["blocks"] == 2000
