"""Autotuner for the compositor: tile size and Gaussian batch depth.

The compositor's cost is dominated by (pixel, splat) evaluations, and a splat
is evaluated for every pixel of every tile its screen box touches, so the best
tile size depends on the splats' screen size: small splats favour small tiles
(fewer wasted evaluations) at the price of more intersections to sort, large
splats the reverse.  The batch depth (splats staged in shared memory per
batch) trades barrier count against shared memory per CTA and thus residency.

`autotune_compositor` times one forward + backward per candidate (tile size,
batch depth) on the caller's own inputs (CUDA events on the current stream)
and caches the winner under a key of the workload's shape, so later calls
with the same shape reuse it.  Tile sizes are those the kernels support (8,
16, 32); depths default to half, one and two times the tile's pixel count,
within the kernels' 32..1024.
"""
from __future__ import annotations

import statistics
from typing import Callable, Dict, Hashable, Iterable, List, Optional, Tuple

import torch

SUPPORTED_TILE_SIZES = (8, 16, 32)
_CACHE: Dict[Hashable, Tuple[int, int]] = {}


def depth_candidates(tile_size: int) -> List[int]:
    px = tile_size * tile_size
    return sorted({max(32, px // 2), px, min(1024, 2 * px)})


def _time(run: Callable[[], None], repeats: int) -> float:
    run()  # warm-up: allocator growth, first-use costs
    samples = []
    for _ in range(repeats):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        run()
        b.record()
        b.synchronize()
        samples.append(a.elapsed_time(b))
    return statistics.median(samples)


def autotune_compositor(key: Hashable, run: Callable[[int, int], None], tiles: Iterable[int] = SUPPORTED_TILE_SIZES,
                        depths: Optional[Iterable[int]] = None, repeats: int = 2
                        ) -> Tuple[Tuple[int, int], Dict[str, float]]:
    """Returns ((tile size, batch depth), {"tile/depth": median ms}).

    `run(tile_size, batch_depth)` must perform the work to be timed (e.g. one
    forward + backward of the renderer) on the current CUDA stream.  `depths`
    (if given) replaces the per-tile default candidates.
    """
    if key in _CACHE:
        return _CACHE[key], {}
    times: Dict[Tuple[int, int], float] = {}
    for ts in tiles:
        if ts not in SUPPORTED_TILE_SIZES:
            continue
        for d in (list(depths) if depths is not None else depth_candidates(ts)):
            times[(ts, d)] = _time(lambda: run(ts, d), repeats)
    best = min(times, key=times.get)
    _CACHE[key] = best
    return best, {f"{t}/{d}": round(v, 3) for (t, d), v in times.items()}


def autotune_tile_size(key: Hashable, run: Callable[[int], None], candidates: Iterable[int] = SUPPORTED_TILE_SIZES,
                       repeats: int = 2) -> Tuple[int, Dict[int, float]]:
    """Tile size only, at each tile's default batch depth: (best, {tile: ms})."""
    (ts, _), times = autotune_compositor(("tile",) + (key if isinstance(key, tuple) else (key,)),
                                         lambda t, d: run(t), tiles=candidates, depths=[0], repeats=repeats)
    return ts, {int(k.split("/")[0]): v for k, v in times.items()}


def clear_cache() -> None:
    _CACHE.clear()
