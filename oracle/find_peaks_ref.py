"""Test infrastructure (oracle): a plain-Python restatement of the peak
finding of the reference's parameter-exploration score.

The reference scores each trace of its exploration run with
scipy.signal.find_peaks(dvdt, 15, distance=5) on dvdt = numpy.diff(v) / dt
and takes the count (GUI/plot_param_explor.py:77-107).  scipy is a
third-party dependency the reference does not vendor (its GUI/requirements.txt
lists it without a pin); the version here is 1.18.  This module restates
the algorithm scipy documents for find_peaks with `height` and `distance`:

  1. local maxima: x[i-1] < x[i], then a run of samples equal to x[i] and a
     smaller sample after it; the peak is the run's middle sample
     ((first + last) // 2); the first and last samples never peak;
  2. keep peaks with x >= height;
  3. visit peaks by decreasing height and drop every peak closer than
     `distance` samples to one that is kept.  scipy orders the visit with
     numpy's argsort, which leaves the order of equal heights unspecified;
     here equal heights visit the later peak first (a stable ascending sort
     read from the end).

It is the checker of the CUDA kernel (tests only); the tests pin it against
scipy itself on inputs without equal-height peak ties.
"""
from __future__ import annotations

import numpy as np


def local_maxima(x) -> list[int]:
    x = [float(e) for e in x]
    out = []
    i, i_max = 1, len(x) - 1
    while i < i_max:
        if x[i - 1] < x[i]:
            ia = i + 1
            while ia < i_max and x[ia] == x[i]:
                ia += 1
            if x[ia] < x[i]:
                out.append((i + ia - 1) // 2)
                i = ia
        i += 1
    return out


def find_peaks(x, height: float, distance: int) -> list[int]:
    """Peak indices of x (steps 1-3 above), ascending."""
    x = np.asarray(x, dtype=np.float64)
    peaks = [p for p in local_maxima(x) if x[p] >= height]
    if distance < 1:
        raise ValueError("distance must be >= 1")
    order = sorted(range(len(peaks)), key=lambda k: (x[peaks[k]], peaks[k]), reverse=True)
    keep = [True] * len(peaks)
    for j in order:
        if not keep[j]:
            continue
        k = j - 1
        while k >= 0 and peaks[j] - peaks[k] < distance:
            keep[k] = False
            k -= 1
        k = j + 1
        while k < len(peaks) and peaks[k] - peaks[j] < distance:
            keep[k] = False
            k += 1
    return [p for p, kp in zip(peaks, keep) if kp]


def dvdt_peak_count(v, dt: float, height: float = 15.0, distance: int = 5) -> int:
    """The score of one trace: peaks of diff(v) / dt, v read as float64."""
    dvdt = np.diff(np.asarray(v, dtype=np.float64)) / dt
    return len(find_peaks(dvdt, height, distance))
