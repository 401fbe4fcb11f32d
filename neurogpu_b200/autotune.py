"""Launch-shape autotuner for the simulation kernels.

Per morphology and batch shape it picks the CTA's warp count and the number
of work items per warp, i.e. how finely the tree is split for the CTA's warps
(more warps or items: more parallel items, better balance and more skeleton
nodes; fewer: longer items).  The candidates
are timed on the device with CUDA events over a short advance of the real
batch (all instances resident, so occupancy matches the production run), and
the fastest is cached per (morphology, n_sets, n_stim, precision).

Fixed by design rather than tuned: one lane per instance and 32 instances per
CTA (the layout that keeps every state access a coalesced 128-byte row), and
the recording cadence, which the caller sets from the output resolution it
needs (ngpu_sim_set_recording's rec_every).
"""
from __future__ import annotations

import hashlib
import json
from pathlib import Path

import numpy as np

from .model import CellModel
from .sim import Model, Simulator

_CACHE: dict[str, dict] = {}


def _key(cell: CellModel, n_sets: int, n_stim: int, precision: str) -> str:
    h = hashlib.sha1()
    for arr in (cell.parent, cell.a, cell.b, cell.cm, cell.mech_mask, cell.section):
        h.update(np.ascontiguousarray(arr).tobytes())
    return f"{h.hexdigest()[:16]}:{n_sets}:{n_stim}:{precision}"


def tune_warps(model: Model | CellModel, params, amps, dts, stim_node: int, stim_area: float, rec_nodes,
               v_init: float, candidates=(2, 4, 6, 8), steps: int = 100, warmup: int = 20,
               precision: str = "fp32", cache_file: str | Path | None = None, items=(2, 3, 4)) -> dict:
    """Times each candidate (warp count, items per warp) on this batch and
    returns {"n_warps": W, "items_per_warp": k, "ms_per_step": {"W:k": ms}}.
    params [n_sets, ...] and amps [n_stim, nt >= warmup + steps] are the
    batch's own inputs."""
    import torch
    model = model if isinstance(model, Model) else Model(model)
    cell = model.cell
    n_sets, n_stim = int(np.asarray(params).shape[0]), int(np.asarray(amps).shape[0])
    key = _key(cell, n_sets, n_stim, precision) + ":" + ",".join(map(str, sorted(items)))
    if cache_file and Path(cache_file).exists() and not _CACHE:
        _CACHE.update(json.loads(Path(cache_file).read_text()))
    if key in _CACHE:
        return _CACHE[key]
    nt = np.asarray(amps).shape[1]
    if nt < warmup + steps:
        raise ValueError(f"need at least {warmup + steps} stimulus steps to time")
    stream = torch.cuda.current_stream()
    timings = {}
    shapes = [(W, k) for W in sorted({int(w) for w in candidates if 1 <= int(w) <= 8})
              for k in (sorted({int(i) for i in items if 1 <= int(i) <= 8}) if W > 1 else [1])]
    for W, k in shapes:
        sim = Simulator(model, n_sets, n_stim, precision, n_warps=W, items_per_warp=k)
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
        timings[(W, k)] = e0.elapsed_time(e1) / steps
        sim.close()
    best = min(timings, key=timings.get)
    res = {"n_warps": best[0], "items_per_warp": best[1],
           "ms_per_step": {f"{w}:{k}": v for (w, k), v in timings.items()}}
    _CACHE[key] = res
    if cache_file:
        Path(cache_file).write_text(json.dumps(_CACHE, indent=1))
    return res
