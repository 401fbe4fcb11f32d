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


def numpy_cell_run(cell, amps, dts, stim_node: int, stim_area: float, rec_nodes, v_init: float, node_fn):
    """FP64 numpy statement of one instance's run: the step of the FP64 oracle
    (oracle/oracle.c run_instance, the reference's U/CudaStuff.cu:227-330) on
    `cell`'s tree, with the channel update of node i given by
    node_fn(i, init, v, dt, states) -> (states, I, G) (init: states at steady
    state for v; otherwise the state update over dt at v; then the current I
    and conductance G at v with the new states).  amps [nt] nA.  Returns V at
    rec_nodes before each step's update, [n_rec, nt]."""
    par = np.asarray(cell.parent)
    a = np.asarray(cell.a, dtype=np.float64)
    b = np.asarray(cell.b, dtype=np.float64)
    cm = np.asarray(cell.cm, dtype=np.float64)
    n = par.size
    nt = len(amps)
    V = np.full(n, float(v_init))
    st, cur, cond = [None] * n, np.zeros(n), np.zeros(n)
    for i in range(n):
        st[i], cur[i], cond[i] = node_fn(i, True, float(v_init), float(dts[0]), None)
    out = np.zeros((len(rec_nodes), nt))
    for t in range(nt):
        dt = float(dts[t])
        out[:, t] = V[rec_nodes]
        rhs = -cur.copy()
        rhs[stim_node] += 100.0 * float(amps[t]) / stim_area
        d = cond + cm / (dt * 1000.0)
        for i in range(1, n):
            dv = V[par[i]] - V[i]
            rhs[i] -= a[i] * dv
            rhs[par[i]] += b[i] * dv
        for i in range(n - 1, 0, -1):  # leaf -> root, excess form
            p = par[i]
            di = d[i] - a[i]
            d[p] += -b[i] * (d[i] / di)
            rhs[p] += -b[i] * (rhs[i] / di)
            d[i] = di
        rhs[0] /= d[0]
        for i in range(1, n):
            rhs[i] = (rhs[i] - a[i] * rhs[par[i]]) / d[i]
        V += rhs
        for i in range(n):
            st[i], cur[i], cond[i] = node_fn(i, False, V[i], dt, st[i])
    return out
