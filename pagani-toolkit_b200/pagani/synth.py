"""Seeded synthetic BOLD series.

No public dataset is named for this path, and the 25,218-voxel subjects of
the reference's timing logs are not distributed, so seeded synthetic series
with the stated shapes stand in for them:

    x_i(t) = AR(1) noise (phi = 0.5, unit innovations, 50-sample burn-in)
             + sum_f L_if s_f(t),   L_if ~ N(0, 0.3^2),  s_f(t) ~ N(0, 1)

drawn from numpy's PCG64 and returned as float32, time-major T x N (the
BOLD[l*N + i] layout the reference gathers from the NIfTI volume).
"""
from __future__ import annotations

import numpy as np

BASE_SEED = 20261203


def subject_seed(config: int, subject: int = 0) -> int:
    return BASE_SEED + config * 1000 + subject


def bold_series(N: int, T: int, n_signals: int, seed: int, phi: float = 0.5,
                loading_sd: float = 0.3, burn_in: int = 50) -> np.ndarray:
    """Return a float32 array of shape (T, N)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    x = np.empty((T, N), np.float32)
    state = rng.standard_normal(N, dtype=np.float32)
    for _ in range(burn_in):
        state = phi * state + rng.standard_normal(N, dtype=np.float32)
    L = (rng.standard_normal((n_signals, N), dtype=np.float32) * loading_sd) if n_signals else None
    S = rng.standard_normal((T, n_signals), dtype=np.float32) if n_signals else None
    for t in range(T):
        state = phi * state + rng.standard_normal(N, dtype=np.float32)
        x[t] = state
    if n_signals:
        x += S @ L
    return x


def roi_batch(n_graphs: int, n_min: int, n_max: int, T: int, n_signals: int, seed: int):
    """Node counts uniform in [n_min, n_max] and one (T, n) series per graph."""
    rng = np.random.Generator(np.random.PCG64(seed))
    sizes = rng.integers(n_min, n_max + 1, size=n_graphs)
    return [bold_series(int(n), T, n_signals, seed + 17 * (g + 1)) for g, n in enumerate(sizes)]
