"""Autotuner for the batched step's work-item shape.

A work item of the batched kernel is one CTA tile marching a segment of
planes.  Two tile shapes are compiled: 8 rows x 128 columns (one warp per
row) and 16 rows x 64 columns (half a warp per row, less idle width when Nz
is small).  Short segments give more items (better balance across SMs for
uneven batches) but repeat the segment warm-up (3 extra planes in, 2 out per
segment); long segments do the opposite.  ``tune_segment`` times the batched
step on a calibration mix of rooms for each (tile, depth) candidate (depth 0
= one wave of items per room) and returns the fastest.  Results are cached
per GPU name in a JSON file next to this module (or at
``$FDTD_B200_TUNE_CACHE``).
"""
from __future__ import annotations

import json
import os
import time
from typing import Dict, Sequence

CANDIDATES = (0, 16, 32, 64, 128)
TILES = (128, 64)
CACHE = os.environ.get("FDTD_B200_TUNE_CACHE",
                       os.path.join(os.path.dirname(os.path.abspath(__file__)), "_tuned.json"))


def _gpu_key() -> str:
    import torch
    return torch.cuda.get_device_name(torch.cuda.current_device())


def _load() -> Dict[str, dict]:
    try:
        with open(CACHE) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def calibration_rooms(n: int = 12, seed: int = 21):
    from .serving import mixed_room_requests
    return [r.room for r in mixed_room_requests(n, seed=seed, steps=(200, 200))]


def time_segment(rooms, planes: int, steps: int = 64, reps: int = 3, tile_k: int = 128) -> float:
    """Seconds per batched step of the calibration mix with the given tile and depth."""
    import torch
    from .serving import EngineBatch, make_solver
    solvers = [make_solver(r) for r in rooms]
    b = EngineBatch()
    b.set_segment(planes)
    b.set_tile(tile_k)
    b.set(solvers, [10 ** 9] * len(solvers))
    b.step(steps, True)          # capture + warm up
    b.sync()
    best = float("inf")
    for _ in range(reps):
        t0 = time.perf_counter()
        b.step(steps, True)
        b.sync()
        best = min(best, (time.perf_counter() - t0) / steps)
    b.set([], [])
    for s in solvers:
        s.close()
    del b
    torch.cuda.synchronize()
    return best


def tune_segment(rooms=None, candidates: Sequence[int] = CANDIDATES, tiles: Sequence[int] = TILES,
                 use_cache: bool = True) -> dict:
    key = _gpu_key()
    cache = _load()
    if use_cache and key in cache and "segment" in cache[key] and "tile" in cache[key]:
        return cache[key]
    rooms = rooms or calibration_rooms()
    timings = {f"{t}x{p}": time_segment(rooms, int(p), tile_k=int(t)) for t in tiles for p in candidates}
    best = min(timings, key=timings.get)
    tile, seg = (int(v) for v in best.split("x"))
    entry = {"tile": tile, "segment": seg, "timings_s_per_step": timings,
             "cells": int(sum(r.cells for r in rooms))}
    cache[key] = entry
    try:
        with open(CACHE, "w") as f:
            json.dump(cache, f, indent=1)
    except OSError:
        pass
    return entry
