"""Autotuner for the PCG kernels' launch shapes.

The SpMV+dot kernels run one warp per 32-row slice with a grid-stride loop; the grid size
trades occupancy and tail effects against the number of reduction partials.  The mixed
form's vector update (y += alpha p, r -= alpha Ap, r.r) strides over the rows four at a time
with its own grid.  For each operator size class the tuner times the engine's own resident
kernels (CUDA events over live launches, ``gipb200_dns_kernel_time``) for a few grid sizes
(multiples of the SM count): first the SpMV grid, then, in the mixed form, the update's
grid, and keeps the fastest of each.  The slice height (32 rows, one warp) and the block
(256 threads) are fixed by the sliced layout and the reductions.  Results are cached per
(kernel, rows, nnz) in memory and, if ``path`` is given, in a JSON file.

For a batch solved by the persistent launch (``tune_batch``) the tuner times whole batch
steps for each launch shape -- threads per CTA (128, 256, 512), rows per warp pass (32:
one slice per warp; 64: two slices in flight) and resident threads per SM (1024 or 1536,
the register budget the kernel is compiled for) -- keeps the fastest, then re-splits the
CTAs by the measured work (rows times the iterations of the last steps) and keeps that
split if it is faster.
"""
from __future__ import annotations

import json
import os

import numpy as np
from typing import Dict, Optional, Sequence

_CACHE: Dict[str, dict] = {}


def _sm_count() -> int:
    import torch
    return torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count


def _best(engine, kernel: str, grids, reps: int, apply) -> tuple:
    timings = {}
    for g in grids:
        apply(g)
        ms, _ = engine.kernel_time(kernel, reps=reps)
        timings[g] = ms
    return min(timings, key=timings.get), timings


def tune(engine, kernel: str = "mixed", rows: int = 0, nnz: int = 0,
         multiples: Sequence[int] = (1, 2, 4, 6, 8), reps: int = 15,
         path: Optional[str] = None) -> dict:
    """Pick the SpMV grid (and in the mixed form the update grid) for `engine` (a
    DnsEngine) and apply them."""
    key = f"{kernel}:{rows}:{nnz}"
    if path and os.path.exists(path) and not _CACHE:
        _CACHE.update(json.load(open(path)))
    if key in _CACHE:
        c = _CACHE[key]
        engine.set_launch(c["blocks"], c.get("vec_blocks", 0))
        return dict(c, cached=True)
    sm = _sm_count()
    grids = sorted({min(8192, m * sm) for m in multiples})
    spmv, t_spmv = _best(engine, kernel, grids, reps, lambda g: engine.set_launch(g, 0))
    out = {"blocks": spmv}
    timings = {"spmv": t_spmv}
    if kernel == "mixed":
        vec, t_vec = _best(engine, "mixed_update", grids, reps,
                           lambda g: engine.set_launch(spmv, g))
        out["vec_blocks"] = vec
        timings["update"] = t_vec
    engine.set_launch(out["blocks"], out.get("vec_blocks", 0))
    _CACHE[key] = out
    if path:
        with open(path, "w") as f:
            json.dump(_CACHE, f)
    return dict(out, cached=False, ms=timings)


BATCH_SHAPES = tuple((b, r, o) for o in (1024, 1536) for r in (32, 64) for b in (128, 256, 512))


def tune_batch(batch, stream, shapes: Sequence = BATCH_SHAPES, steps: int = 2) -> dict:
    """Pick the persistent solve's launch shape and CTA split for `batch` (a DnsBatch) by
    timing `steps` whole batch steps per candidate (the instances advance meanwhile)."""
    import torch

    def timed():
        batch.advance(1, stream)  # capture outside the timed steps
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        batch.advance(steps, stream)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / steps

    ms = {}
    for shape in shapes:
        batch.set_solver(True, *shape)
        ms[tuple(shape)] = timed()
    best = min(ms, key=ms.get)
    batch.set_solver(True, *best)
    t_default = timed()
    rows = np.array([e.n_inner for e in batch.instances], np.float64)
    iters = np.array([max(float(np.mean(e.history()["iters"][-steps:])), 1.0)
                      for e in batch.instances])
    weights = rows * iters
    batch.balance(weights)
    t_measured = timed()
    balanced = t_measured < t_default
    if not balanced:
        batch.balance(None)
    return {"block": best[0], "rows_per_warp": best[1],
            "threads_per_sm": best[2] if len(best) > 2 else 1024,
            "balanced_by_iterations": balanced,
            "weights": weights.tolist() if balanced else None,
            "ms": {"x".join(str(v) for v in k): round(t, 3) for k, t in ms.items()},
            "ms_default_split": round(t_default, 3), "ms_measured_split": round(t_measured, 3)}
