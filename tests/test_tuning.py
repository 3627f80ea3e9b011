"""CPU checks of the compositor autotuner's host logic (textured_gaussians_b200/
tuning.py) with its CUDA-event timer replaced by a table of costs: the fastest
(tile size, batch depth) candidate wins, the winner is cached per workload key
(later calls time nothing), unsupported tile sizes are skipped, and the
default depth candidates stay within the kernels' 32..1024.
"""
import pytest

from textured_gaussians_b200 import tuning


@pytest.fixture
def fake_timer(monkeypatch):
    calls = []
    costs = {}

    def _time(run, repeats):
        run()
        return costs[calls[-1]]

    monkeypatch.setattr(tuning, "_time", _time)
    tuning.clear_cache()
    yield calls, costs
    tuning.clear_cache()


def test_depth_candidates():
    assert tuning.depth_candidates(8) == [32, 64, 128]
    assert tuning.depth_candidates(16) == [128, 256, 512]
    assert tuning.depth_candidates(32) == [512, 1024]


def test_fastest_candidate_wins_and_is_cached(fake_timer):
    calls, costs = fake_timer
    for ts in (8, 16, 32):
        for d in tuning.depth_candidates(ts):
            costs[(ts, d)] = 10.0 + ts + d / 100
    costs[(16, 256)] = 1.0
    run = lambda ts, d: calls.append((ts, d))  # noqa: E731
    best, times = tuning.autotune_compositor(("shape", 1), run)
    assert best == (16, 256)
    assert len(times) == len(calls) == 8 and times["16/256"] == 1.0
    n = len(calls)
    best2, times2 = tuning.autotune_compositor(("shape", 1), run)
    assert best2 == best and times2 == {} and len(calls) == n  # cached: nothing timed again
    best3, _ = tuning.autotune_compositor(("shape", 2), run)    # another workload is tuned afresh
    assert best3 == (16, 256) and len(calls) == 2 * n


def test_unsupported_tiles_are_skipped_and_depths_override(fake_timer):
    calls, costs = fake_timer
    costs.update({(8, 64): 3.0, (16, 64): 2.0})
    best, times = tuning.autotune_compositor("k", lambda ts, d: calls.append((ts, d)), tiles=(8, 12, 16),
                                             depths=[64])
    assert best == (16, 64) and sorted(calls) == [(8, 64), (16, 64)] and set(times) == {"8/64", "16/64"}


def test_tile_only_form(fake_timer):
    calls, costs = fake_timer
    costs.update({(8, 0): 5.0, (16, 0): 4.0, (32, 0): 6.0})
    best, times = tuning.autotune_tile_size("k", lambda ts: calls.append((ts, 0)))
    assert best == 16 and times == {8: 5.0, 16: 4.0, 32: 6.0}
