"""Seeded synthetic request streams for the serving path.

The serving configuration: Poisson arrivals; each request 1..64 volumes with a
log-uniform count; cube side L from {6, 8, 12, 16, 17, 24, 36} with probability
proportional to 1/L; forward / inverse 50/50; complex128 75% / complex64 25%;
re/im uniform[-1, 1).
"""
from __future__ import annotations

import numpy as np

SIDES = (6, 8, 12, 16, 17, 24, 36)


def request_stream(n: int, rate_hz: float, seed: int = 2024):
    """n requests: list of dicts with arrival time `t` (seconds from 0),
    `shape`, `batch`, `direction` (-1/+1) and `precision` (0 c128, 1 c64)."""
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
    return [{"t": float(t[k]), "shape": (int(sides[k]),) * 3, "batch": int(counts[k]),
             "direction": int(direction[k]), "precision": int(precision[k])} for k in range(n)]


def volume_bytes(req) -> int:
    e = 16 if req["precision"] == 0 else 8
    return int(np.prod(req["shape"])) * e * req["batch"]
