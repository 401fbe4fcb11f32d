"""Shared test helpers: spike times and error summaries."""
from __future__ import annotations

import numpy as np


def spike_times(v: np.ndarray, dt: float, thresh: float = -20.0) -> np.ndarray:
    """Upward threshold crossings of a 1-D trace, linearly interpolated (ms)."""
    v = np.asarray(v, dtype=np.float64)
    i = np.nonzero((v[:-1] < thresh) & (v[1:] >= thresh))[0]
    frac = (thresh - v[i]) / (v[i + 1] - v[i])
    return (i + frac) * dt


def spike_time_error(a: np.ndarray, b: np.ndarray, dt: float, thresh: float = -20.0) -> tuple[float, int]:
    """Max |t_a - t_b| over matched spikes of traces [..., nt]; and the number
    of traces whose spike counts differ."""
    a2 = a.reshape(-1, a.shape[-1])
    b2 = b.reshape(-1, b.shape[-1])
    worst, mismatched = 0.0, 0
    for x, y in zip(a2, b2):
        sx, sy = spike_times(x, dt, thresh), spike_times(y, dt, thresh)
        if sx.size != sy.size:
            mismatched += 1
            continue
        if sx.size:
            worst = max(worst, float(np.max(np.abs(sx - sy))))
    return worst, mismatched


def subthreshold_error(a: np.ndarray, b: np.ndarray, dt: float, window_ms: float = 2.0,
                       thresh: float = -20.0) -> float:
    """max |a - b| over samples farther than window_ms from any spike of either trace."""
    a2 = a.reshape(-1, a.shape[-1]).astype(np.float64)
    b2 = b.reshape(-1, b.shape[-1]).astype(np.float64)
    w = int(round(window_ms / dt))
    worst = 0.0
    for x, y in zip(a2, b2):
        keep = np.ones(x.size, dtype=bool)
        for tr in (x, y):
            for t in spike_times(tr, dt, thresh):
                k = int(t / dt)
                keep[max(0, k - w):k + w + 1] = False
        if keep.any():
            worst = max(worst, float(np.max(np.abs(x[keep] - y[keep]))))
    return worst
