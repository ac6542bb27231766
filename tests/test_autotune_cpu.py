"""The launch-shape autotuner's selection and cache logic, on the host (fake engine)."""
import json

from gip_b200 import autotune


class FakeEngine:
    """Times each kernel's grid size from a table, records the launches it was given."""

    def __init__(self, ms_by_blocks, ms_update=None):
        self.ms = ms_by_blocks
        self.ms_update = ms_update or {}
        self.blocks = self.vec = None
        self.timed = []

    def set_launch(self, blocks, vec):
        self.blocks, self.vec = blocks, vec

    def kernel_time(self, kernel, reps=15):
        if kernel == "mixed_update":
            self.timed.append(("update", self.vec))
            return self.ms_update[self.vec], 0.0
        self.timed.append(("spmv", self.blocks))
        return self.ms[self.blocks], 0.0


def test_picks_fastest_grids_and_caches(tmp_path, monkeypatch):
    monkeypatch.setattr(autotune, "_sm_count", lambda: 148)
    monkeypatch.setattr(autotune, "_CACHE", {})
    ms = {148: 1.0, 296: 0.7, 592: 0.5, 888: 0.6, 1184: 0.9}
    mu = {148: 0.4, 296: 0.3, 592: 0.35, 888: 0.2, 1184: 0.25}
    E = FakeEngine(ms, mu)
    path = str(tmp_path / "tune.json")
    r = autotune.tune(E, "mixed", rows=1000, nnz=7000, path=path)
    assert (r["blocks"], r["vec_blocks"]) == (592, 888) and not r["cached"]
    assert (E.blocks, E.vec) == (592, 888)
    assert sorted(b for k, b in E.timed if k == "spmv") == sorted(ms)
    assert sorted(b for k, b in E.timed if k == "update") == sorted(mu)
    assert json.load(open(path)) == {"mixed:1000:7000": {"blocks": 592, "vec_blocks": 888}}
    # the same operator class again: no timing, the cached grids applied
    F = FakeEngine(ms, mu)
    r = autotune.tune(F, "mixed", rows=1000, nnz=7000, path=path)
    assert r["cached"] and F.timed == [] and (F.blocks, F.vec) == (592, 888)
    # a fresh process reads the file
    monkeypatch.setattr(autotune, "_CACHE", {})
    G = FakeEngine(ms, mu)
    assert autotune.tune(G, "mixed", rows=1000, nnz=7000, path=path)["cached"]
    assert G.timed == [] and (G.blocks, G.vec) == (592, 888)


def test_grid_capped_and_classes_separate(monkeypatch):
    monkeypatch.setattr(autotune, "_sm_count", lambda: 2000)
    monkeypatch.setattr(autotune, "_CACHE", {})
    E = FakeEngine({2000: 0.3, 4000: 0.2, 8192: 0.25})
    r = autotune.tune(E, "fp64", rows=5, nnz=9, multiples=(1, 2, 8, 16))
    assert max(b for _, b in E.timed) == 8192 and r["blocks"] == 4000
    assert "vec_blocks" not in r                 # the FP64 forms tune the SpMV grid only
    E2 = FakeEngine({2000: 0.1, 4000: 0.2, 8192: 0.25})
    assert autotune.tune(E2, "fp64", rows=6, nnz=9, multiples=(1, 2, 8))["blocks"] == 2000


class FakeBatch:
    """A batch whose step time depends on the persistent launch shape and the CTA split."""

    class Inst:
        def __init__(self, n, iters):
            self.n_inner, self._it = n, iters

        def history(self):
            import numpy as np
            return {"iters": np.array([self._it] * 4)}

    def __init__(self, ms_by_shape, ms_balanced):
        self.ms, self.ms_bal = ms_by_shape, ms_balanced
        self.shape, self.weights = None, None
        self.instances = [self.Inst(1000, 50), self.Inst(8000, 120)]

    def set_solver(self, persistent, block, rpw, occ=1024):
        self.shape = (block, rpw)

    def balance(self, w):
        self.weights = None if w is None else list(w)

    def advance(self, n, stream=None):
        pass


def test_tune_batch_picks_shape_and_split(monkeypatch):
    import types
    ms = {(128, 32): 3.0, (256, 32): 2.0, (512, 32): 2.5, (128, 64): 2.8, (256, 64): 1.5,
          (512, 64): 1.9}
    B = FakeBatch(ms, 1.2)
    clock = {"t": 0.0}

    class Ev:
        def __init__(self, enable_timing=True):
            self.t = 0.0

        def record(self, stream=None):
            clock["t"] += B.ms_bal if B.weights else B.ms[B.shape]
            self.t = clock["t"]

        def synchronize(self):
            pass

        def elapsed_time(self, other):
            return (other.t - self.t) * 2  # two timed steps

    fake_torch = types.SimpleNamespace(cuda=types.SimpleNamespace(Event=Ev))
    monkeypatch.setitem(__import__("sys").modules, "torch", fake_torch)
    shapes = [(b, r, 1024) for (b, r) in ms]
    r = autotune.tune_batch(B, None, shapes=shapes, steps=2)
    assert (r["block"], r["rows_per_warp"]) == (256, 64) and B.shape == (256, 64)
    assert r["balanced_by_iterations"] and B.weights == [1000 * 50.0, 8000 * 120.0]
    assert r["weights"] == [1000 * 50.0, 8000 * 120.0]
    B2 = FakeBatch(ms, 9.0)  # the measured split is slower: the default split is restored
    B = B2
    r = autotune.tune_batch(B2, None, shapes=shapes, steps=2)
    assert not r["balanced_by_iterations"] and B2.weights is None and r["weights"] is None
