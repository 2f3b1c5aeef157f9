"""Seeded synthetic series for the benchmark workloads.

The reference measures on the user's own nanopore / UCR data; no public
suite exists for this path, so the workloads are seeded synthetic signals
with the shapes, lengths and value distributions the benchmark configurations
name.  Every generator takes an explicit seed; the default seeds are
0x0DBA0000 + configuration number.

* ``random_walks``     -- Gaussian random walk, step sigma 1 (plain DBA workload).
* ``nanopore_like``    -- piecewise-constant current levels ~ N(90, 12) pA with
  geometric dwell lengths and additive Gaussian noise (medoid, stripe,
  batched and serving workloads).
"""
from __future__ import annotations

import numpy as np

SEED_BASE = 0x0DBA0000


def _lengths(rng: np.random.Generator, n: int, lo: int, hi: int) -> np.ndarray:
    return rng.integers(lo, hi + 1, size=n, dtype=np.int64)


def random_walks(n: int, lo: int, hi: int, seed: int, dtype=np.float32) -> list[np.ndarray]:
    """n Gaussian random walks with lengths uniform in [lo, hi]."""
    rng = np.random.default_rng(seed)
    lens = _lengths(rng, n, lo, hi)
    return [np.cumsum(rng.standard_normal(int(L))).astype(dtype) for L in lens]


def step_signal(rng: np.random.Generator, L: int, level_mu: float, level_sd: float,
                dwell_mean: float, noise_sd: float) -> np.ndarray:
    """One piecewise-constant signal with geometric dwells plus Gaussian noise."""
    out = np.empty(L, dtype=np.float64)
    pos = 0
    p = 1.0 / dwell_mean
    while pos < L:
        dwell = int(rng.geometric(p))
        level = rng.normal(level_mu, level_sd)
        out[pos:pos + dwell] = level
        pos += dwell
    out += rng.normal(0.0, noise_sd, size=L)
    return out


def nanopore_like(n: int, lo: int, hi: int, seed: int, dwell_mean: float = 10.0,
                  noise_sd: float = 2.0, dtype=np.float32) -> list[np.ndarray]:
    """n nanopore-like step signals with lengths uniform in [lo, hi]."""
    rng = np.random.default_rng(seed)
    lens = _lengths(rng, n, lo, hi)
    return [step_signal(rng, int(L), 90.0, 12.0, dwell_mean, noise_sd).astype(dtype) for L in lens]


def medoid_workload(n_series: int = 2000, len_lo: int = 2000, len_hi: int = 8000,
                    seed: int = SEED_BASE + 2) -> list[np.ndarray]:
    """The medoid all-vs-all workload (2000 series by default): lengths uniform
    in [len_lo, len_hi], piecewise-constant N(90, 12) pA levels with geometric
    dwells of mean 10 samples plus N(0, 2) noise, float32, sorted by length as
    performDBA sorts before its medoid pass (dba.hpp:876-885).  Raw values:
    z-normalisation is the pipeline's first device step."""
    rng = np.random.default_rng(seed)
    lens = rng.integers(len_lo, len_hi + 1, size=n_series)
    series = []
    for L in lens:
        dw = rng.geometric(0.1, size=int(L) // 4 + 16)
        while dw.sum() < L:
            dw = np.concatenate([dw, rng.geometric(0.1, size=int(L) // 4 + 16)])
        levels = rng.normal(90.0, 12.0, size=len(dw))
        x = np.repeat(levels, dw)[:L] + rng.normal(0.0, 2.0, size=int(L))
        series.append(x.astype(np.float32))
    series.sort(key=len)
    return series


def znorm_host(series: list[np.ndarray]) -> list[np.ndarray]:
    """Population z-normalisation in float64, cast back to each series' dtype.

    Used only to prepare benchmark inputs that are already normalised; the
    library's own z-normalisation kernel is what the pipeline runs."""
    out = []
    for s in series:
        x = s.astype(np.float64)
        sd = x.std()
        out.append(((x - x.mean()) / (sd if sd != 0 else 1.0)).astype(s.dtype))
    return out


def step_signals(rng: np.random.Generator, lens, level_mu: float, level_sd: float,
                 dwell_mean: float, noise_sd: float, dtype=np.float32):
    """Vectorised step_signal for many (long) series: geometric dwells with the
    given mean, N(level_mu, level_sd) levels, N(0, noise_sd) noise."""
    out = []
    p = 1.0 / dwell_mean
    for L in lens:
        L = int(L)
        dw = rng.geometric(p, size=int(L / dwell_mean * 1.1) + 16)
        while dw.sum() < L:
            dw = np.concatenate([dw, rng.geometric(p, size=int(L / dwell_mean * 0.2) + 16)])
        levels = rng.normal(level_mu, level_sd, size=len(dw))
        x = np.repeat(levels, dw)[:L] + rng.normal(0.0, noise_sd, size=L)
        out.append(x.astype(dtype))
    return out
