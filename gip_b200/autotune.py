"""Autotuner for the PCG kernels' launch shape.

The SpMV+dot kernels run one warp per 32-row slice with a grid-stride loop; the grid size
trades occupancy and tail effects against the number of reduction partials.  For each
operator size class the tuner times the engine's own resident kernel (CUDA events over
live launches, ``gipb200_dns_kernel_time``) for a few grid sizes (multiples of the SM
count) and keeps the fastest.  Results are cached per (kernel, rows, nnz) in memory and,
if ``path`` is given, in a JSON file.
"""
from __future__ import annotations

import json
import os
from typing import Dict, Optional, Sequence

_CACHE: Dict[str, int] = {}


def _sm_count() -> int:
    import torch
    return torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count


def tune(engine, kernel: str = "mixed", rows: int = 0, nnz: int = 0,
         multiples: Sequence[int] = (1, 2, 4, 6, 8), reps: int = 15,
         path: Optional[str] = None) -> dict:
    """Pick the SpMV grid for `engine` (a DnsEngine) and apply it."""
    key = f"{kernel}:{rows}:{nnz}"
    if path and os.path.exists(path) and not _CACHE:
        _CACHE.update(json.load(open(path)))
    if key in _CACHE:
        engine.set_launch(_CACHE[key], 0)
        return {"blocks": _CACHE[key], "cached": True}
    sm = _sm_count()
    timings = {}
    for m in multiples:
        blocks = min(8192, m * sm)
        engine.set_launch(blocks, 0)
        ms, _ = engine.kernel_time(kernel, reps=reps)
        timings[blocks] = ms
    best = min(timings, key=timings.get)
    engine.set_launch(best, 0)
    _CACHE[key] = best
    if path:
        with open(path, "w") as f:
            json.dump(_CACHE, f)
    return {"blocks": best, "cached": False, "ms": timings}
