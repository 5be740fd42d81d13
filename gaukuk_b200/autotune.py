"""Tile-shape autotuner for the fused 2D stage kernel.

The stage kernel's tile is (threads per CTA, rows per segment): a CTA of T
threads updates T-4 columns and marches up R rows.  Narrow, short tiles give
more CTAs (better for small grids), wide, long ones less halo work.  The
tuner measures rather than models: it times a few device-resident steps for
each candidate with CUDA events on the library's stream and keeps the
fastest.

* ``tune_single(sim)``: one problem; sets the winner with gk_set_tiling.
* ``tune_ensemble(ens)``: threads first (one value for the whole persistent
  launch), then rows per grid-size class, coordinate-wise.

Winners are cached by (grid shape(s), arithmetic mode) in
``lib/tiling_cache.json`` next to the built library.
"""
from __future__ import annotations

import json
import os
from typing import Dict, List, Sequence, Tuple

THREADS = (64, 128, 256)
ROWS = (4, 8, 16, 32)
_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "tiling_cache.json")


def _load_cache() -> Dict[str, object]:
    try:
        with open(_CACHE) as f:
            return json.load(f)
    except Exception:
        return {}


def _save_cache(c: Dict[str, object]) -> None:
    try:
        os.makedirs(os.path.dirname(_CACHE), exist_ok=True)
        with open(_CACHE, "w") as f:
            json.dump(c, f, indent=1, sort_keys=True)
    except OSError:
        pass


def _time_ms(stream_ptr: int, fn, steps: int) -> float:
    import torch
    st = torch.cuda.ExternalStream(stream_ptr)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    fn(steps)
    e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1) / steps


def tune_single(sim, steps: int = 6, use_cache: bool = True) -> Tuple[int, int, float]:
    """Best (threads, rows) for one problem; applied to `sim`.  Runs
    (1 + steps) x 12 steps of the problem (its state advances)."""
    key = f"single:{sim.params.nx}x{sim.params.ny}:{sim.mode}"
    cache = _load_cache() if use_cache else {}
    if key in cache:
        th, rows, ms = cache[key]
        sim.set_tiling(th, rows)
        return th, rows, ms
    best = None
    for th in THREADS:
        for rows in ROWS:
            sim.set_tiling(th, rows)
            sim.run_steps(1)  # builds the graph for this shape
            ms = _time_ms(sim.stream, sim.enqueue_steps, steps)
            if best is None or ms < best[2]:
                best = (th, rows, ms)
    sim.set_tiling(best[0], best[1])
    cache[key] = list(best)
    _save_cache(cache)
    return best


def tune_ensemble(ens, steps: int = 4, use_cache: bool = True) -> Dict[str, object]:
    """Best threads and rows-per-size-class for an ensemble; applied to it.
    Each trial runs 1 + steps ensemble steps (the states advance)."""
    sizes = [(s.params.nx, s.params.ny) for s in ens.sims]
    classes = sorted(set(sizes))
    key = "ens:" + ",".join(f"{a}x{b}:{sizes.count((a, b))}" for a, b in classes) + \
        f":{ens.sims[0].mode}"
    cache = _load_cache() if use_cache else {}
    if key in cache:
        r = cache[key]
        ens.set_tiling(r["threads"], [r["rows"][f"{a}x{b}"] for a, b in sizes])
        return r
    stream = ens.info()["stream"]

    def trial(th: int, rows_by_class: Dict[Tuple[int, int], int]) -> float:
        ens.set_tiling(th, [rows_by_class[s] for s in sizes])
        ens.run_steps(1)
        return _time_ms(stream, ens.enqueue_steps, steps)

    rows_by_class = {c: 16 for c in classes}
    best_th, best_ms = None, None
    for th in THREADS:
        ms = trial(th, rows_by_class)
        if best_ms is None or ms < best_ms:
            best_th, best_ms = th, ms
    for c in classes:
        for r in ROWS:
            cand = dict(rows_by_class)
            cand[c] = r
            ms = trial(best_th, cand)
            if ms < best_ms:
                best_ms, rows_by_class = ms, cand
    ens.set_tiling(best_th, [rows_by_class[s] for s in sizes])
    result = {"threads": best_th, "rows": {f"{a}x{b}": rows_by_class[(a, b)] for a, b in classes},
              "ms_per_step": best_ms}
    cache[key] = result
    _save_cache(cache)
    return result
