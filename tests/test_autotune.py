"""The autotuner's search logic and sampling (CPU; the renderer is faked)."""
import pytest

from ymrt_b200 import autotune


def test_points_cover_the_space_in_fixed_order():
    space = {"b": [1, 2], "a": [10, 20, 30]}
    pts = autotune.points(space)
    assert len(pts) == 6
    assert pts[0] == {"a": 10, "b": 1} and pts[-1] == {"a": 30, "b": 2}
    assert autotune.points(space) == pts


def test_search_picks_the_fastest_and_skips_failures():
    cost = {(1 << 20, 0): 5.0, (1 << 20, 1): 3.0, (1 << 21, 0): 4.0, (1 << 21, 1): 9.0}
    calls = []

    def measure(p):
        calls.append(p)
        if p["queue_capacity"] == 1 << 21 and p["sort_hits"] == 1:
            raise RuntimeError("rejected")
        return cost[(p["queue_capacity"], p["sort_hits"])]

    r = autotune.search({"queue_capacity": [1 << 20, 1 << 21], "sort_hits": [0, 1]}, measure, repeats=2)
    assert r["best"] == {"queue_capacity": 1 << 20, "sort_hits": 1}
    assert r["ms"] == 3.0
    assert sum(1 for t in r["table"] if t["ms"] is None) == 1
    # one warm-up and two timed calls per point (the failing point stops at its first)
    assert len(calls) == 3 * 3 + 1


def test_search_fails_when_nothing_runs():
    def measure(p):
        raise RuntimeError("no device")

    with pytest.raises(RuntimeError):
        autotune.search({"sort_hits": [0, 1]}, measure)


def test_sample_band_fills_waves_or_takes_the_frame():
    b, e = autotune.sample_tiles(1920, 1080, 64, 1 << 21, waves=4)
    assert 0 < b < e < 120 * 68
    assert (e - b) * 256 * 64 >= 4 * (1 << 21)
    assert autotune.sample_tiles(256, 256, 16, 1 << 21) == (0, 0)  # whole frame is smaller
