"""Tile-size autotuner for the compositor.

The compositor's cost is dominated by (pixel, splat) evaluations, and a
splat is evaluated for every pixel of every tile its screen box touches, so
the best tile size depends on the splats' screen size: small splats favour
small tiles (fewer wasted evaluations) at the price of more intersections to
sort.  `autotune_tile_size` times one forward + backward per candidate on the
caller's own inputs (CUDA events on the current stream) and caches the winner
under a key of the workload's shape, so later calls with the same shape reuse
it.  Candidates are the tile sizes the kernels support (8 and 16).
"""
from __future__ import annotations

import statistics
from typing import Callable, Dict, Hashable, Iterable, Tuple

import torch

SUPPORTED_TILE_SIZES = (8, 16)
_CACHE: Dict[Hashable, int] = {}


def autotune_tile_size(key: Hashable, run: Callable[[int], None], candidates: Iterable[int] = SUPPORTED_TILE_SIZES,
                       repeats: int = 2) -> Tuple[int, Dict[int, float]]:
    """Returns (best tile size, {tile size: median ms}).

    `run(tile_size)` must perform the work to be timed (e.g. one forward +
    backward of the renderer) on the current CUDA stream.
    """
    if key in _CACHE:
        return _CACHE[key], {}
    times: Dict[int, float] = {}
    for ts in candidates:
        if ts not in SUPPORTED_TILE_SIZES:
            continue
        run(ts)  # warm-up: allocator growth, first-use costs
        samples = []
        for _ in range(repeats):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            run(ts)
            b.record()
            b.synchronize()
            samples.append(a.elapsed_time(b))
        times[ts] = statistics.median(samples)
    best = min(times, key=times.get)
    _CACHE[key] = best
    return best, times


def clear_cache() -> None:
    _CACHE.clear()
