"""The tile autotuner's host logic (gaukuk_b200/autotune.py) on fake problems
with a fake device timer: the single-problem search keeps the fastest
(threads, rows) of the full grid and applies it; the ensemble search picks
threads at 16 rows, then rows class by class; winners are cached by shape,
instance counts and mode, and a cached winner is applied without timing."""
import json
from types import SimpleNamespace

import pytest

from gaukuk_b200 import autotune


class FakeSim:
    def __init__(self, nx, ny, mode="fast"):
        self.params = SimpleNamespace(nx=nx, ny=ny)
        self.mode = mode
        self.stream = 0
        self.tiling = None
        self.calls = []

    def set_tiling(self, threads, rows):
        self.tiling = (threads, rows)
        self.calls.append(self.tiling)

    def run_steps(self, n):
        return n

    def enqueue_steps(self, n):
        pass


class FakeEnsemble:
    def __init__(self, sizes, mode="fast"):
        self.sims = [FakeSim(a, b, mode) for a, b in sizes]
        self.tiling = None

    def info(self):
        return {"stream": 0}

    def set_tiling(self, threads, rows):
        self.tiling = (threads, list(rows))

    def run_steps(self, n):
        return n

    def enqueue_steps(self, n):
        pass


@pytest.fixture
def cache(tmp_path, monkeypatch):
    path = tmp_path / "tiling_cache.json"
    monkeypatch.setattr(autotune, "_CACHE", str(path))
    return path


def _timer(monkeypatch, cost, target):
    """_time_ms replaced by cost(target's current tiling); returns the call log."""
    log = []

    def fake(stream, fn, steps):
        log.append(target.tiling)
        return cost(target.tiling)

    monkeypatch.setattr(autotune, "_time_ms", fake)
    return log


def test_single_search_keeps_the_fastest_and_caches_it(cache, monkeypatch):
    sim = FakeSim(256, 256)
    best = (64, 8)
    log = _timer(monkeypatch, lambda t: 1.0 + abs(t[0] - best[0]) / 64 + abs(t[1] - best[1]) / 8, sim)
    th, rows, ms = autotune.tune_single(sim)
    assert (th, rows) == best and ms == 1.0
    assert sim.tiling == best
    assert len(log) == len(autotune.THREADS) * len(autotune.ROWS)
    saved = json.loads(cache.read_text())
    assert saved["single:256x256:fast"] == [64, 8, 1.0]

    # the cached winner is applied without timing; another mode is a new key
    sim2 = FakeSim(256, 256)
    log.clear()
    assert autotune.tune_single(sim2)[:2] == best and sim2.tiling == best and log == []
    sim3 = FakeSim(256, 256, mode="parity")
    log3 = _timer(monkeypatch, lambda t: 2.0, sim3)
    autotune.tune_single(sim3)
    assert len(log3) == len(autotune.THREADS) * len(autotune.ROWS)
    assert set(json.loads(cache.read_text())) == {"single:256x256:fast", "single:256x256:parity"}


def test_single_search_ties_keep_the_first_candidate(cache, monkeypatch):
    sim = FakeSim(128, 128)
    _timer(monkeypatch, lambda t: 1.0, sim)
    th, rows, _ = autotune.tune_single(sim, use_cache=False)
    assert (th, rows) == (autotune.THREADS[0], autotune.ROWS[0])


def test_ensemble_search_threads_then_rows_per_class(cache, monkeypatch):
    sizes = [(128, 128), (512, 512), (128, 128), (256, 256)]
    ens = FakeEnsemble(sizes)
    want_rows = {(128, 128): 4, (256, 256): 8, (512, 512): 32}

    def cost(t):
        th, rows = t
        c = 1.0 + (0.0 if th == 128 else 0.5)
        for s, r in zip(sizes, rows):
            c += 0.01 * abs(r - want_rows[s]) / 4
        return c

    log = _timer(monkeypatch, cost, ens)
    r = autotune.tune_ensemble(ens)
    assert r["threads"] == 128
    assert r["rows"] == {"128x128": 4, "256x256": 8, "512x512": 32}
    assert ens.tiling == (128, [want_rows[s] for s in sizes])
    # threads are timed at 16 rows in every class
    assert [t for t, _ in log[:len(autotune.THREADS)]] == list(autotune.THREADS)
    assert all(rows == [16] * len(sizes) for _, rows in log[:len(autotune.THREADS)])
    assert len(log) == len(autotune.THREADS) + 3 * len(autotune.ROWS)
    key = "ens:128x128:2,256x256:1,512x512:1:fast"
    assert json.loads(cache.read_text())[key]["threads"] == 128

    ens2 = FakeEnsemble(sizes)
    log.clear()
    autotune.tune_ensemble(ens2)
    assert log == [] and ens2.tiling == ens.tiling
