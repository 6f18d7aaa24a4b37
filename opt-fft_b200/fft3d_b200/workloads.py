"""Seeded synthetic request streams for the serving path.

The serving configuration: Poisson arrivals; each request 1..64 volumes with a
log-uniform count; cube side L from {6, 8, 12, 16, 17, 24, 36} with probability
proportional to 1/L; forward / inverse 50/50; complex128 75% / complex64 25%;
re/im uniform[-1, 1).
"""
from __future__ import annotations

import numpy as np

SIDES = (6, 8, 12, 16, 17, 24, 36)


def request_arrays(n: int, rate_hz: float, seed: int = 2024):
    """The stream as arrays: arrival time t (seconds from 0), side L, volume
    count, direction (-1/+1) and precision (0 c128, 1 c64) of each request."""
    rng = np.random.default_rng(seed)
    p = np.array([1.0 / L for L in SIDES])
    p /= p.sum()
    sides = rng.choice(SIDES, size=n, p=p)
    counts = np.floor(np.exp(rng.uniform(0.0, np.log(65.0), n))).astype(int)
    counts = np.clip(counts, 1, 64)
    direction = np.where(rng.random(n) < 0.5, -1, +1)
    precision = np.where(rng.random(n) < 0.75, 0, 1)
    gaps = rng.exponential(1.0 / rate_hz, n) if rate_hz > 0 else np.zeros(n)
    t = np.cumsum(gaps) - (gaps[0] if n else 0.0)
    return {"t": t, "side": sides.astype(np.int64), "batch": counts.astype(np.int64),
            "direction": direction.astype(np.int64), "precision": precision.astype(np.int64)}


def request_stream(n: int, rate_hz: float, seed: int = 2024):
    """n requests: list of dicts with arrival time `t` (seconds from 0),
    `shape`, `batch`, `direction` (-1/+1) and `precision` (0 c128, 1 c64)."""
    a = request_arrays(n, rate_hz, seed)
    return [{"t": float(a["t"][k]), "shape": (int(a["side"][k]),) * 3, "batch": int(a["batch"][k]),
             "direction": int(a["direction"][k]), "precision": int(a["precision"][k])}
            for k in range(n)]


def arena_offsets(nbytes, arena_bytes):
    """Byte offset of each request's buffer in a rotating arena: requests take
    consecutive ranges in arrival order and wrap to the start when the next one
    would run past the end, so a stream far larger than the arena cycles
    through it (a request never straddles the end)."""
    nbytes = np.asarray(nbytes, dtype=np.int64)
    if len(nbytes) and int(nbytes.max()) > arena_bytes:
        raise ValueError("a request is larger than the arena")
    start = np.empty_like(nbytes)
    pos = 0
    for k, b in enumerate(nbytes.tolist()):
        if pos + b > arena_bytes:
            pos = 0
        start[k] = pos
        pos += b
    return start


def volume_bytes(req) -> int:
    e = 16 if req["precision"] == 0 else 8
    return int(np.prod(req["shape"])) * e * req["batch"]
