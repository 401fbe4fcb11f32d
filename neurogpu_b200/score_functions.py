"""Trace-comparison scores of the reference's GA driver (GUI/score_functions.py),
restated with numpy.

Every function keeps the reference's name and signature
``f(target, data, dt=0.1, stims=None, index=None) -> float`` and its
arithmetic, quirks included (listed per function), so a GA written against
the reference scores identically.  ``stims``/``index`` only keyed a result
cache in the reference (the helpers' three-way results); here the helpers
are cheap enough to recompute, so the arguments are accepted and ignored.

``score_batch`` evaluates one function over many traces at once, which is
how the B200 driver scores a whole population.
"""
from __future__ import annotations

import math
from typing import Callable, Sequence

import numpy as np

threshold = -10   # peak threshold of traj_score_single_peak (score_functions.py:10)


# ---- utilities (score_functions.py:14-41) -------------------------------------------------
def zero_pad(list1, list2):
    """Pads the shorter list with zeros; scalars pass through unchanged."""
    if isinstance(list1, (int, float)) or isinstance(list2, (int, float)):
        return list1, list2
    list1, list2 = list(list1), list(list2)
    if len(list1) > len(list2):
        list2 = list2 + [0] * (len(list1) - len(list2))
    elif len(list2) > len(list1):
        list1 = list1 + [0] * (len(list2) - len(list1))
    return list1, list2


def safe_mean(lis):
    """Mean, or 0 for an empty input."""
    if np.size(lis) == 0:
        return 0
    return np.mean(lis)


def find_positive_inds(lis):
    return [int(i) for i in np.nonzero(np.asarray(lis) > 0)[0]]


def find_peaks(lis, min_value):
    """Interior samples >= both neighbours and >= min_value (plateaus give one
    index per sample); returns (values, indices)."""
    x = np.asarray(lis)
    if x.size < 3:
        return [], []
    mid = x[1:-1]
    inds = np.nonzero((mid >= x[:-2]) & (mid >= x[2:]) & (mid >= min_value))[0] + 1
    return [x[i] for i in inds], [int(i) for i in inds]


def diff(lis):
    x = np.asarray(lis)
    return list(x[1:] - x[:-1])


# ---- pointwise scores (:45-65) ---------------------------------------------------------------
def chi_square_normal(target, data, dt=0.1, stims=None, index=None):
    """mean((target - data)^2)."""
    return safe_mean(np.square(np.array(target) - np.array(data)))


def abs_cumsum_diff(target, data, dt=0.1, stims=None, index=None):
    """mean |cumsum(target) - cumsum(data)|."""
    return safe_mean(np.absolute(np.cumsum(np.array(target)) - np.cumsum(np.array(data))))


def comp_rest_potential(target, data, dt=0.1, stims=None, index=None):
    """Squared difference of the last samples (the resting potential after
    the protocol)."""
    k = len(target) - 1
    return (target[k] - data[k]) ** 2


# ---- action-potential widths (:69-130) ----------------------------------------------------------
def _positive_runs(x):
    """(starts, ends) of runs of consecutive samples > 0 (ends inclusive)."""
    pos = np.nonzero(np.asarray(x) > 0)[0]
    if pos.size == 0:
        return None
    brk = np.nonzero(np.diff(pos) > 1)[0]
    starts = np.concatenate(([pos[0]], pos[brk + 1]))
    ends = np.concatenate((pos[brk], [pos[-1]]))
    return starts, ends


def comp_width_helper(target, data):
    """[sum of squared width differences over zero-padded per-AP widths,
    squared difference of the mean widths]; widths in samples, an AP being a
    run of samples above 0 mV."""
    rt, rd = _positive_runs(target), _positive_runs(data)
    wt = [int(e - s) for s, e in zip(*rt)] if rt is not None else []
    wd = [int(e - s) for s, e in zip(*rd)] if rd is not None else []
    at = safe_mean(wt) if rt is not None else 0
    ad = safe_mean(wd) if rd is not None else 0
    if rt is not None or rd is not None:
        wt, wd = zero_pad(wt, wd)
    else:
        wt, wd, at, ad = [], [], 0, 0
    return [sum((wt[i] - wd[i]) ** 2 for i in range(len(wd))), (at - ad) ** 2]


def comp_width(target, data, dt=0.1, stims=None, index=None):
    return comp_width_helper(target, data)[0]


def comp_width_avg(target, data, dt=0.1, stims=None, index=None):
    return comp_width_helper(target, data)[1]


# ---- action-potential heights (:134-189) -------------------------------------------------------
def comp_height_helper(target, data):
    """[sum of squared differences of zero-padded peak heights, squared
    difference of the mean heights].  Peaks: find_peaks(., 0.1), taken only
    when the trace has a positive sample; heights are measured from the last
    sample, and a zero-padded missing peak counts as height -V_last (the
    reference's arithmetic)."""
    pt = find_peaks(target, 0.1)[0] if np.any(np.asarray(target) > 0) else []
    pd_ = find_peaks(data, 0.1)[0] if np.any(np.asarray(data) > 0) else []
    pt, pd_ = zero_pad(pt, pd_)
    k = len(target) - 1
    vt, vd = target[k], data[k]
    ht = [p - vt for p in pt]
    hd = [p - vd for p in pd_]
    at = safe_mean(np.array(ht)) if len(ht) > 0 else 0
    ad = safe_mean(np.array(hd)) if len(hd) > 0 else 0
    return [sum((ht[i] - hd[i]) ** 2 for i in range(len(ht))), (at - ad) ** 2]


def comp_height(target, data, dt=0.1, stims=None, index=None):
    return comp_height_helper(target, data)[0]


def comp_height_avg(target, data, dt=0.1, stims=None, index=None):
    return comp_height_helper(target, data)[1]


# ---- phase-plane trajectory scores (:192-263) --------------------------------------------------
_V_EDGES = np.linspace(-80, 70, 100)
_DV_EDGES = np.linspace(-6, 40, 100)


def traj_score_helper(target, data):
    """[rms difference of the normalised (V, dV) histograms, max and mean
    absolute difference of their normalised 2-D cumulative sums] over
    99 x 99 bins spanning V in [-80, 70] mV, dV in [-6, 40] mV per sample."""
    t = np.asarray(target, dtype=np.float64)
    d = np.asarray(data, dtype=np.float64)
    edges = [_V_EDGES, _DV_EDGES]
    ht = np.histogram2d(t[1:], t[1:] - t[:-1], bins=edges)[0]
    with np.errstate(divide="ignore", invalid="ignore"):
        ct = np.cumsum(np.cumsum(ht, axis=0), axis=1)
        ct = ct / ct.max()
        ht = ht / ht.sum()
        hd = np.histogram2d(d[1:], d[1:] - d[:-1], bins=edges)[0]
        hd = hd / hd.sum()
        t_score = np.mean(np.mean((ht - hd) ** 2, axis=1))
        cd = np.cumsum(np.cumsum(hd, axis=0), axis=1)
        cd = cd / cd.max()
    cdiff = np.abs(cd - ct)
    return [t_score ** 0.5, np.max(cdiff), np.mean(np.mean(cdiff, axis=1))]


def traj_score_1(target, data, dt=0.1, stims=None, index=None):
    return traj_score_helper(target, data)[0]


def traj_score_2(target, data, dt=0.1, stims=None, index=None):
    return traj_score_helper(target, data)[1]


def traj_score_3(target, data, dt=0.1, stims=None, index=None):
    return traj_score_helper(target, data)[2]


# ---- inter-spike intervals (:266-290) ----------------------------------------------------------
def isi(target, data, dt=0.1, stims=None, index=None):
    """rms difference of the zero-padded peak-time lists (peaks >= 0 mV,
    times dt, 2dt, ...), normalised by the rms of the target's successive
    peak-time differences (1 when that is 0); NaN scores 0."""
    times = np.cumsum(np.full(len(target), dt, dtype=np.float64))
    pt = [times[j] for j in find_peaks(target, 0)[1]]
    pd_ = [times[j] for j in find_peaks(data, 0)[1]]
    pt, pd_ = zero_pad(pt, pd_)
    score = safe_mean([(pt[j] - pd_[j]) ** 2 for j in range(len(pt))]) ** 0.5
    norm = safe_mean([e ** 2 for e in diff(pt)]) ** 0.5
    if not norm or norm == 0:
        norm = 1
    out = float(safe_mean(score)) / norm
    return 0 if np.isnan(out) else out


# ---- vector similarity (:293-323) --------------------------------------------------------------
def rev_dot_product(target, data, dt=0.1, stims=None, index=None):
    """1 - cos(angle between target and data)."""
    t, d = np.array(target), np.array(data)
    return 1 - (float(np.dot(t, d)) / (np.sqrt(np.sum(np.square(t))) * np.sqrt(np.sum(np.square(d)))))


def KL_divergence(target, data, dt=0.1, stims=None, index=None):
    """sum q log(q / p) over samples where both are nonzero, with p, q the
    traces shifted by |min| + 0.1 and normalised to sum 1 (target -> p)."""
    def prob(v):
        v = np.array(v)
        v = v + np.absolute(np.amin(v)) + 0.1
        return v / float(np.sum(v))
    p, q = prob(target), prob(data)
    m = (p != 0) & (q != 0)
    # the reference sums term by term in float64; math.fsum would round differently
    d = 0
    for a, b in zip(p[m], q[m]):
        d += float(b) * np.log(float(b) / a)
    return d


# ---- per-peak phase-plane score (:326-411) ----------------------------------------------------
def traj_score_single_peak(target, data, dt=0.1, stims=None, index=None):
    """rms over peaks (>= -10 mV, NaN-padded to a common count) of the
    difference of 100 x 100 (V, dV/dt) histograms of a window around each
    peak, the half window being the smaller of 25 ms and half the distance
    to the neighbouring peaks.  Like the reference it needs at least two
    peaks in each trace (IndexError otherwise) and slices with Python's
    negative-index semantics near the trace start."""
    n_x = n_y = 100

    def nan_pad(a, b):
        if len(a) > len(b):
            b = b + [math.nan] * (len(a) - len(b))
        elif len(b) > len(a):
            a = a + [math.nan] * (len(b) - len(a))
        return a, b

    def pairs(peaks, max_half_ms):
        out = []
        max_half = max_half_ms / dt
        for i in range(len(peaks)):
            half = max_half
            if i == 0:
                w = (peaks[i + 1] - peaks[i]) / 2
            elif i == len(peaks) - 1 or math.isnan(peaks[i + 1]):
                w = (peaks[i] - peaks[i - 1]) / 2
            else:
                w = min((peaks[i + 1] - peaks[i]) / 2, (peaks[i] - peaks[i - 1]) / 2)
            if w < half:
                half = w
            out.append((peaks[i], math.floor(half)))
        return out

    def plane(signal, pair):
        p, half = pair
        if math.isnan(p):
            return [math.nan], [math.nan]
        seg = signal[p - half:p + half]
        return seg[1:], np.array(diff(seg)) / np.array([dt] * (len(seg) - 1)).tolist()

    tp = find_peaks(target, threshold)[1]
    dp = find_peaks(data, threshold)[1]
    tp, dp = nan_pad(tp, dp)
    tpairs, dpairs = pairs(tp, 25), pairs(dp, 25)
    total = 0
    for i in range(len(tp)):
        tx, ty = plane(target, tpairs[i])
        dx, dy = plane(data, dpairs[i])
        xb = np.linspace(np.nanmin([min(tx), min(dx)]), np.nanmax([max(tx), max(dx)]), n_x + 1)
        yb = np.linspace(np.nanmin([min(ty), min(dy)]), np.nanmax([max(ty), max(dy)]), n_y + 1)
        ht = np.histogram2d(tx, ty, bins=(xb, yb))[0]
        hd = np.histogram2d(dx, dy, bins=(xb, yb))[0]
        total += np.sum((ht - hd) ** 2)
    return (total / (n_x * n_y)) ** 0.5


# ---- dynamic time warping (:414-427) -----------------------------------------------------------
def DTWDistance(target, data, dt=0.1, stims=None, index=None):
    """Dynamic time warping with |x - y| cost.  The reference returns the
    cell (len(target) - 1, len(data) - 1) of the (len + 1)-square table,
    i.e. the warping cost of the traces without their last samples, divided
    by len(target); kept as is.  Computed by anti-diagonals (each cell's
    value is the same expression of the same operands)."""
    t = np.asarray(target, dtype=np.float64)
    d = np.asarray(data, dtype=np.float64)
    n, m = t.size, d.size
    D = np.full((n + 1, m + 1), np.inf)
    D[0, 0] = 0.0
    for s in range(2, n + m + 1):
        i = np.arange(max(1, s - m), min(n, s - 1) + 1)
        j = s - i
        cost = np.abs(t[i - 1] - d[j - 1])
        D[i, j] = cost + np.minimum(np.minimum(D[i - 1, j], D[i, j - 1]), D[i - 1, j - 1])
    return D[n - 1, m - 1] / n


FUNCTIONS: dict[str, Callable] = {f.__name__: f for f in (
    chi_square_normal, abs_cumsum_diff, comp_rest_potential, comp_width, comp_width_avg, comp_height,
    comp_height_avg, traj_score_1, traj_score_2, traj_score_3, isi, rev_dot_product, KL_divergence,
    traj_score_single_peak, DTWDistance)}


def score_batch(name: str, target: Sequence[float], traces: np.ndarray, dt: float = 0.1) -> np.ndarray:
    """One score of every row of traces [n, nt] against target [nt].  The
    pointwise scores are vectorised over the batch; the rest run per trace."""
    traces = np.asarray(traces, dtype=np.float64)
    t = np.asarray(target, dtype=np.float64)
    if name == "chi_square_normal":
        return np.mean(np.square(t[None, :] - traces), axis=1)
    if name == "abs_cumsum_diff":
        return np.mean(np.abs(np.cumsum(t)[None, :] - np.cumsum(traces, axis=1)), axis=1)
    if name == "comp_rest_potential":
        return (t[-1] - traces[:, -1]) ** 2
    f = FUNCTIONS[name]
    return np.array([f(t, row, dt) for row in traces], dtype=np.float64)
