"""Launch-shape and recording autotuner for the simulation kernels.

Per morphology and batch shape it picks:

* the layout: one lane per instance with 32 instances per CTA (every state
  access a coalesced 128-byte row; fills a B200 from a few thousand
  instances on), or one warp per instance (the instance's tree split over
  the warp's lanes; spreads a small batch over every SM);
* the CTA shape of the chosen layout: warps per CTA and work items per warp
  (lane layout), or instances per CTA and work items per instance (warp
  layout) -- how finely the tree is split: more items balance better and
  cost more skeleton nodes;
* the recording cadence: the coarsest sampling of the traces at which the
  caller's measures (spike times, spike peaks) stay within its tolerances,
  judged on a pilot run recorded every step.

Candidates are timed on the device with CUDA events over a short advance of
the real batch (all instances resident, so occupancy matches the production
run); the fastest is cached per (morphology, n_sets, n_stim, precision).
"""
from __future__ import annotations

import hashlib
import json
from pathlib import Path

import numpy as np

from .model import CellModel
from .sim import Model, Simulator

_CACHE: dict[str, dict] = {}

# candidate shapes: (warps per CTA, items per warp) of the lane layout and
# (instances per CTA, items per instance) of the warp layout
LANE_SHAPES = ((2, 2), (4, 2), (4, 3), (6, 3), (8, 2), (8, 3), (8, 4))
# lane-layout CTAs of more than 8 warps, timed for batches of at most one
# 32-instance group per SM (compiled then for one CTA per SM)
WIDE_SHAPES = ((12, 2), (12, 3), (16, 2), (16, 3))
SM_COUNT = 148
WARP_SHAPES = ((1, 16), (1, 32), (1, 64), (2, 32), (4, 32), (8, 32))
# the warp layout is timed up to this many instances (beyond, 32 instances
# per CTA fill every SM several times over and the lane layout's coalesced
# rows win)
WARP_LAYOUT_MAX_INSTANCES = 148 * 32 * 2


def _key(cell: CellModel, n_sets: int, n_stim: int, precision: str) -> str:
    h = hashlib.sha1()
    for arr in (cell.parent, cell.a, cell.b, cell.cm, cell.mech_mask, cell.section):
        h.update(np.ascontiguousarray(arr).tobytes())
    return f"{h.hexdigest()[:16]}:{n_sets}:{n_stim}:{precision}"


def _time_shape(model: Model, n_sets, n_stim, precision, layout, W, k, params, amps, dts, stim_node, stim_area,
                rec_nodes, v_init, steps, warmup, stream) -> float:
    import torch
    sim = Simulator(model, n_sets, n_stim, precision, n_warps=W, items_per_warp=k, layout=layout)
    try:
        sim.set_params(params)
        sim.set_stimulus(amps, dts, stim_node, stim_area)
        sim.set_recording(rec_nodes)
        sim.init(v_init, stream)
        sim.advance(0, warmup, stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sim.advance(warmup, steps, stream)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps
    finally:
        sim.close()


def tune(model: Model | CellModel, params, amps, dts, stim_node: int, stim_area: float, rec_nodes,
         v_init: float, steps: int = 100, warmup: int = 20, precision: str = "fp32",
         lane_shapes=LANE_SHAPES, warp_shapes=WARP_SHAPES, cache_file: str | Path | None = None) -> dict:
    """Times every candidate layout and shape on this batch and returns
    {"layout": "lane" | "warp", "n_warps": W, "items_per_warp": k,
    "ms_per_step": {"lane:W:k" | "warp:W:k": ms}}, ready for
    Simulator(..., layout=, n_warps=, items_per_warp=).  params [n_sets, ...]
    and amps [n_stim, nt >= warmup + steps] are the batch's own inputs."""
    import torch
    model = model if isinstance(model, Model) else Model(model)
    cell = model.cell
    n_sets, n_stim = int(np.asarray(params).shape[0]), int(np.asarray(amps).shape[0])
    if lane_shapes is LANE_SHAPES and (n_sets * n_stim + 31) // 32 <= SM_COUNT:
        lane_shapes = LANE_SHAPES + WIDE_SHAPES
    lane_shapes = tuple((int(w), int(k)) for w, k in lane_shapes if 1 <= int(w) <= 16 and 1 <= int(k) <= 8)
    warp_shapes = tuple((int(w), int(k)) for w, k in warp_shapes if 1 <= int(w) <= 8 and 1 <= int(k) <= 512)
    if n_sets * n_stim > WARP_LAYOUT_MAX_INSTANCES:
        warp_shapes = ()
    key = (_key(cell, n_sets, n_stim, precision) + ":layout:" + ",".join(f"{w}.{k}" for w, k in lane_shapes) + "/" +
           ",".join(f"{w}.{k}" for w, k in warp_shapes))
    _load(cache_file)
    if key in _CACHE:
        return _CACHE[key]
    nt = np.asarray(amps).shape[1]
    if nt < warmup + steps:
        raise ValueError(f"need at least {warmup + steps} stimulus steps to time")
    stream = torch.cuda.current_stream()
    timings = {}
    cands = [("lane", w, k) for w, k in lane_shapes] + [("warp", w, k) for w, k in warp_shapes]
    for layout, W, k in cands:
        timings[(layout, W, k)] = _time_shape(model, n_sets, n_stim, precision, layout, W, k, params, amps, dts,
                                              stim_node, stim_area, rec_nodes, v_init, steps, warmup, stream)
    best = min(timings, key=timings.get)
    res = {"layout": best[0], "n_warps": best[1], "items_per_warp": best[2],
           "ms_per_step": {f"{a}:{w}:{k}": v for (a, w, k), v in timings.items()}}
    _store(key, res, cache_file)
    return res


def tune_warps(model: Model | CellModel, params, amps, dts, stim_node: int, stim_area: float, rec_nodes,
               v_init: float, candidates=(2, 4, 6, 8), steps: int = 100, warmup: int = 20,
               precision: str = "fp32", cache_file: str | Path | None = None, items=(2, 3, 4)) -> dict:
    """The lane layout's shape alone (up to 8 warps: the shapes a batch of
    several morphologies runs): times each (warp count, items per warp) and
    returns {"n_warps": W, "items_per_warp": k, "ms_per_step":
    {"W:k": ms}} (what a batch of several morphologies, which runs the lane
    layout, needs per member)."""
    shapes = [(int(W), int(k)) for W in sorted({int(w) for w in candidates if 1 <= int(w) <= 8})
              for k in (sorted({int(i) for i in items if 1 <= int(i) <= 8}) if W > 1 else [1])]
    cell = model.cell if isinstance(model, Model) else model
    key = (_key(cell, int(np.asarray(params).shape[0]), int(np.asarray(amps).shape[0]), precision) + ":warps:" +
           ",".join(f"{w}.{k}" for w, k in shapes))
    _load(cache_file)
    if key in _CACHE:
        return _CACHE[key]
    r = tune(model, params, amps, dts, stim_node, stim_area, rec_nodes, v_init, steps=steps, warmup=warmup,
             precision=precision, lane_shapes=shapes, warp_shapes=(), cache_file=cache_file)
    res = {"n_warps": r["n_warps"], "items_per_warp": r["items_per_warp"],
           "ms_per_step": {k.split(":", 1)[1]: v for k, v in r["ms_per_step"].items()}}
    _store(key, res, cache_file)
    return res


# --------------------------------------------------------- recording cadence
def _crossings(v: np.ndarray, thresh: float) -> np.ndarray:
    """Upward threshold crossings of one trace, linearly interpolated, in samples."""
    i = np.nonzero((v[:-1] < thresh) & (v[1:] >= thresh))[0]
    return i + (thresh - v[i]) / (v[i + 1] - v[i])


def cadence_errors(traces: np.ndarray, k: int, thresh: float = -20.0) -> dict:
    """What recording every k-th step loses on traces [..., nt] recorded every
    step: the traces whose spike counts change, the largest shift of an
    interpolated spike time (in steps), and the largest drop of a spike's
    peak (mV; the peak is the largest sample between the spike's upward and
    downward crossings)."""
    tr = np.asarray(traces, dtype=np.float64).reshape(-1, np.asarray(traces).shape[-1])
    mism, dt_worst, peak_worst = 0, 0.0, 0.0
    for v in tr:
        full = _crossings(v, thresh)
        sub = _crossings(v[::k], thresh) * k
        if full.size != sub.size:
            mism += 1
            continue
        if full.size:
            dt_worst = max(dt_worst, float(np.max(np.abs(full - sub))))
            down = np.nonzero((v[:-1] >= thresh) & (v[1:] < thresh))[0]
            for s in full:
                e = down[down > s]
                hi = int(e[0]) + 1 if e.size else v.size
                lo = int(s) + 1
                p_full = float(v[lo:hi].max()) if hi > lo else float(v[int(s)])
                seg = v[::k][(lo + k - 1) // k:(hi + k - 1) // k]
                p_sub = float(seg.max()) if seg.size else float(v[(int(s) // k) * k])
                peak_worst = max(peak_worst, p_full - p_sub)
    return {"count_mismatches": mism, "spike_shift_steps": dt_worst, "peak_drop_mV": peak_worst}


def tune_cadence(traces: np.ndarray, dt: float, spike_tol_ms: float = 0.05, peak_tol_mv: float = 1.0,
                 candidates=(1, 2, 4, 5, 8, 10, 20, 40), thresh: float = -20.0) -> dict:
    """The coarsest recording cadence (rec_every, from `candidates`) at which
    traces [..., nt] of a pilot run recorded every step keep every spike,
    move no interpolated spike time by more than spike_tol_ms and lower no
    spike peak by more than peak_tol_mv.  Returns {"rec_every": k,
    "errors": {k: cadence_errors}} for the candidates tried."""
    errors, best = {}, 1
    for k in sorted({int(c) for c in candidates if int(c) >= 1}):
        e = cadence_errors(traces, k, thresh)
        errors[k] = e
        if e["count_mismatches"] == 0 and e["spike_shift_steps"] * dt <= spike_tol_ms and \
                e["peak_drop_mV"] <= peak_tol_mv:
            best = k
        else:
            break
    return {"rec_every": best, "errors": errors}


def _load(cache_file):
    if cache_file and Path(cache_file).exists() and not _CACHE:
        _CACHE.update(json.loads(Path(cache_file).read_text()))


def _store(key, res, cache_file):
    _CACHE[key] = res
    if cache_file:
        Path(cache_file).write_text(json.dumps(_CACHE, indent=1))
