"""The seeded serving stream and the rotating-arena layout (CPU only).

The serving benchmark replays a stream of 1e6 requests whose inputs cycle
through fixed device arenas; these checks cover the host-side generator: the
request distribution matches the serving configuration, the array and dict
forms are the same stream, and arena ranges never run past the arena or
overlap a neighbour.
"""
import numpy as np
import pytest

from fft3d_b200.workloads import SIDES, arena_offsets, request_arrays, request_stream


def test_arrays_and_dicts_are_the_same_stream():
    a = request_arrays(500, rate_hz=1000.0, seed=11)
    d = request_stream(500, rate_hz=1000.0, seed=11)
    for k in (0, 17, 499):
        assert d[k]["shape"] == (int(a["side"][k]),) * 3
        assert d[k]["batch"] == a["batch"][k]
        assert d[k]["direction"] == a["direction"][k]
        assert d[k]["precision"] == a["precision"][k]
        assert d[k]["t"] == pytest.approx(a["t"][k])


def test_stream_distribution():
    a = request_arrays(200_000, rate_hz=1e6, seed=3)
    assert set(np.unique(a["side"])) == set(SIDES)
    p = np.array([1.0 / L for L in SIDES])
    p /= p.sum()
    freq = np.array([(a["side"] == L).mean() for L in SIDES])
    assert np.allclose(freq, p, atol=0.005)
    assert a["batch"].min() == 1 and a["batch"].max() == 64
    assert abs((a["precision"] == 0).mean() - 0.75) < 0.005
    assert abs((a["direction"] == -1).mean() - 0.5) < 0.005
    # Poisson arrivals: exponential gaps with mean 1/rate
    assert np.mean(np.diff(a["t"])) == pytest.approx(1e-6, rel=0.02)


def test_arena_offsets_wrap_without_overlap():
    rng = np.random.default_rng(5)
    nbytes = rng.integers(1, 1000, 5000) * 16
    arena = 100_000
    off = arena_offsets(nbytes, arena)
    assert (off >= 0).all() and (off + nbytes <= arena).all()
    # consecutive requests never overlap (they are in flight together)
    for k in range(1, len(off)):
        if off[k] != 0:
            assert off[k] == off[k - 1] + nbytes[k - 1]
    with pytest.raises(ValueError):
        arena_offsets([arena + 16], arena)
