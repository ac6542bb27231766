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
"""
from __future__ import annotations

import json
import os
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
