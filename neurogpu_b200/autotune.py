"""Launch-shape autotuner for the simulation kernels.

Per morphology and batch shape it picks the CTA's warp count, i.e. how finely
the tree is split into work items for the CTA's warps (more warps: more
parallel items and more skeleton nodes; fewer: longer items).  The candidates
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
               precision: str = "fp32", cache_file: str | Path | None = None) -> dict:
    """Times each candidate warp count on this batch and returns
    {"n_warps": best, "ms_per_step": {W: ms}}.  params [n_sets, ...] and
    amps [n_stim, nt >= warmup + steps] are the batch's own inputs."""
    import torch
    model = model if isinstance(model, Model) else Model(model)
    cell = model.cell
    n_sets, n_stim = int(np.asarray(params).shape[0]), int(np.asarray(amps).shape[0])
    key = _key(cell, n_sets, n_stim, precision)
    if cache_file and Path(cache_file).exists() and not _CACHE:
        _CACHE.update(json.loads(Path(cache_file).read_text()))
    if key in _CACHE:
        return _CACHE[key]
    nt = np.asarray(amps).shape[1]
    if nt < warmup + steps:
        raise ValueError(f"need at least {warmup + steps} stimulus steps to time")
    stream = torch.cuda.current_stream()
    timings = {}
    for W in sorted({int(w) for w in candidates if 1 <= int(w) <= 8}):
        sim = Simulator(model, n_sets, n_stim, precision, n_warps=W)
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
        timings[W] = e0.elapsed_time(e1) / steps
        sim.close()
    best = min(timings, key=timings.get)
    res = {"n_warps": best, "ms_per_step": {str(k): v for k, v in timings.items()}}
    _CACHE[key] = res
    if cache_file:
        Path(cache_file).write_text(json.dumps(_CACHE, indent=1))
    return res
