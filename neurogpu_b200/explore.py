"""Parameter exploration: a grid over two GA parameters, one simulation of
every grid point, and a spike-count score map.

Mirrors the reference's exploration run: GUI/run_neuroGPU.py:15-31 and
GUI/plot_param_explor.py:36-53 (``gen_params``: the base row of
opt_table.csv with parameter 0 swept over linspace(0, 10, 100) and parameter
2 over linspace(0, 20, 100), parameter 0 outermost: 10,000 sets), one
neuroGPU run of all sets, then GUI/plot_param_explor.py:77-107
(``calc_scores``: per trace the number of peaks of dV/dt that
scipy.signal.find_peaks(dvdt, 15, distance=5) finds, as a 100 x 100 map).
Here the sets run as one resident batch and the score is computed on the GPU
where the traces lie (``Simulator.dvdt_peaks``, ``ngpu_sim_dvdt_peaks``);
no VHotP file or trace readback is involved.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path
from typing import Sequence

import numpy as np

from . import _ffi, formats
from .evaluator import allparams_from_mapping

# GUI/plot_param_explor.py:16,33-35
HIGH_NUMBER = 10000
NBINS = 100
DT = 0.1
HEIGHT = 15.0
DISTANCE = 5


def read_opt_table(path: str | Path) -> tuple[list[str], np.ndarray, np.ndarray, np.ndarray]:
    """opt_table.csv: a header of parameter names, then the rows lower bound,
    upper bound and base value (GUI/run_neuroGPU.py:16-20 reads it with
    numpy.genfromtxt(..., names=True)).  Returns (names, lb, ub, base)."""
    lines = [ln for ln in Path(path).read_text().splitlines() if ln.strip()]
    names = [x.strip() for x in lines[0].split(",")]
    rows = [np.array([float(x) for x in ln.split(",") if x.strip()], dtype=np.float64) for ln in lines[1:4]]
    for r in rows:
        if r.size != len(names):
            raise ValueError(f"{path}: a row holds {r.size} values for {len(names)} names")
    return names, rows[0], rows[1], rows[2]


def gen_params(base: Sequence[float], p1: int = 0, p1_values: Sequence[float] | None = None, p2: int = 2,
               p2_values: Sequence[float] | None = None) -> np.ndarray:
    """The exploration grid (GUI/run_neuroGPU.py:15-31): one row per (v1, v2)
    in p1_values x p2_values, parameter p1 outermost, every other parameter at
    its base value.  Defaults: the reference's linspace(0, 10, 100) for
    parameter 0 and linspace(0, 20, 100) for parameter 2."""
    base = np.asarray(base, dtype=np.float64)
    v1 = np.linspace(0, 10, NBINS) if p1_values is None else np.asarray(p1_values, dtype=np.float64)
    v2 = np.linspace(0, 20, NBINS) if p2_values is None else np.asarray(p2_values, dtype=np.float64)
    if not (0 <= p1 < base.size and 0 <= p2 < base.size) or p1 == p2:
        raise ValueError("p1 and p2 must be two different parameter indices")
    out = np.repeat(base[None, :], v1.size * v2.size, axis=0)
    out[:, p1] = np.repeat(v1, v2.size)
    out[:, p2] = np.tile(v2, v1.size)
    return out


def mapping_for(template_row: Sequence[float], n_sections: int, assign: dict) -> tuple:
    """An (template_row, indicator_row, corrections) mapping, as
    ``evaluator.load_mapping`` reads from AllParams_for_params.csv, built
    from a rule instead: assign[k] = (p, sections) marks parameter p
    (param-major AllParams rows: entry p * n_sections + section) in the
    given sections (None: every section where the template's value is
    nonzero) for GA parameter k (indicator 12300 + k,
    T/extractModel_mappings.py:258-272)."""
    from .evaluator import PARAM_INDICATOR_BASE
    tmpl = np.asarray(template_row, dtype=np.float64)
    if tmpl.size % n_sections:
        raise ValueError("the template row is not n_params x n_sections")
    t = tmpl.reshape(-1, n_sections)
    ind = np.zeros_like(t)
    for k, (p, secs) in assign.items():
        where = t[p] != 0 if secs is None else np.isin(np.arange(n_sections), np.asarray(secs))
        ind[p][where] = PARAM_INDICATOR_BASE + int(k)
    return tmpl, ind.reshape(-1), {}


def _as_exact_f32(volts) -> np.ndarray:
    v = np.asarray(volts)
    if v.dtype == np.float32:
        return np.ascontiguousarray(v)
    f = v.astype(np.float32)
    ok = np.isnan(v) | (f.astype(v.dtype) == v)
    if not ok.all():
        raise ValueError("traces must be float32 values (the simulator's; VHotP files hold them as float64)")
    return np.ascontiguousarray(f)


def dvdt_peak_counts(traces, dt: float = DT, height: float = HEIGHT, distance: int = DISTANCE, stream=None):
    """Per trace, the number of peaks scipy.signal.find_peaks(diff(v) / dt,
    height, distance) finds, on the GPU (ngpu_trace_dvdt_peaks).

    traces [n_traces, n_samples]: a float32 CUDA tensor (read in place) or a
    host array of float32 values (float64 holding float32 values, as VHotP
    files do, is accepted).  Returns an int32 CUDA tensor [n_traces]."""
    import torch
    if hasattr(traces, "is_cuda") and traces.is_cuda:
        t = traces if traces.dtype == torch.float32 else None
        if t is None:
            raise ValueError("CUDA traces must be float32")
    else:
        t = torch.from_numpy(_as_exact_f32(traces)).cuda()
    if t.dim() != 2:
        raise ValueError("traces must be [n_traces, n_samples]")
    n, ns = int(t.shape[0]), int(t.shape[1])
    L = _ffi.lib()
    need = int(L.ngpu_dvdt_peaks_scratch_bytes(n, ns))
    scratch = torch.empty(max(need, 4), dtype=torch.uint8, device=t.device)
    out = torch.empty(n, dtype=torch.int32, device=t.device)
    sp = None if stream is None else C.c_void_p(int(getattr(stream, "cuda_stream", stream)))
    _ffi.check("ngpu_trace_dvdt_peaks", L.ngpu_trace_dvdt_peaks(
        C.c_void_p(t.data_ptr()), int(t.stride(0)), int(t.stride(1)), n, ns, float(dt), float(height),
        int(distance), C.c_void_p(scratch.data_ptr()), scratch.numel(), C.c_void_p(out.data_ptr()), sp))
    if stream is None:
        torch.cuda.synchronize()
    return out


def calc_scores(volts, nbins: int = NBINS, dt: float = DT, height: float = HEIGHT,
                distance: int = DISTANCE) -> np.ndarray:
    """The score map of GUI/plot_param_explor.py:77-107: volts is a VHotP
    file (read as the reference reads it, float64 samples) or an array
    holding nbins^2 traces back to back; every trace's dV/dt peak count, as
    an [nbins, nbins] float64 array (first grid parameter along rows).  The
    reference's NaN test on the count never fires (a count is an integer), so
    HIGH_NUMBER never appears here either."""
    v = formats.read_vhot(volts) if isinstance(volts, (str, Path)) else np.asarray(volts)
    psize = nbins * nbins
    v = v.reshape(-1)
    nt = v.size // psize
    if nt < 1:
        raise ValueError(f"{v.size} samples hold no trace for each of the {psize} grid points")
    v = v[:nt * psize].reshape(psize, nt)   # the file's overhang is dropped, as there
    counts = dvdt_peak_counts(v, dt=dt, height=height, distance=distance)
    return counts.cpu().numpy().astype(np.float64).reshape(nbins, nbins)


def grid_simulation(model: "formats.ReferenceModel", mapping: tuple, grid: np.ndarray,
                    stim: np.ndarray | None = None, rec_every: int = 1, precision: str = "fp32",
                    chunk: int = 2000, score_dt: float | None = None):
    """One resident simulation of every row of `grid` (GA parameter vectors;
    their AllParams rows by ``allparams_from_mapping``, mapping as
    ``evaluator.load_mapping`` returns it) under stimulus `stim` ([nt] nA;
    default the model's first), run to the end, recording the model's first
    recording site.  Returns (simulator, score_dt): the trace stays on the
    GPU for ``Simulator.dvdt_peaks``.

    The reference samples every step and divides by its own constant
    dt = 0.1 (GUI/plot_param_explor.py:35, the step of its examples); here
    score_dt defaults to the sample spacing (step dt x rec_every) as the
    shortest decimal that gives its float32 value back, the value times.csv
    holds (0.1, not the float32 0.100000001)."""
    from .sim import Model, Simulator
    rows = allparams_from_mapping(grid, *mapping, dtype=np.float32)
    cell = model.cell
    n_comps = cell.n_sections
    n_file_params = rows.shape[1] // n_comps
    file_params = rows.reshape(len(rows), n_file_params, n_comps)
    n_models = int(model.raw["basic_const"]["NModels"][0]) if model.raw else None
    params = formats.map_params(file_params, n_models, n_file_params) if n_models else file_params
    amps = np.asarray(model.amps[0] if stim is None else stim, dtype=np.float32).reshape(1, -1)
    dts = np.asarray(model.dts, dtype=np.float32)
    if not np.all(dts == dts[0]):
        raise ValueError("the score needs a uniform sample spacing (times.csv holds several dt)")
    sim = Simulator(Model(cell), len(grid), 1, precision)
    sim.set_params(params)
    sim.set_stimulus(amps, dts, model.stim_node, model.stim_area)
    sim.set_recording(np.asarray(model.rec_nodes[:1], dtype=np.int32), rec_every)
    sim.init(model.v_init)
    nt = amps.shape[1]
    for t0 in range(0, nt, chunk):
        sim.advance(t0, min(chunk, nt - t0))
    if score_dt is None:
        score_dt = float(np.format_float_positional(np.float32(dts[0]) * np.float32(rec_every), unique=True))
    return sim, score_dt


def explore(model: "formats.ReferenceModel", mapping: tuple, base: Sequence[float], p1: int = 0,
            p1_values: Sequence[float] | None = None, p2: int = 2, p2_values: Sequence[float] | None = None,
            stim: np.ndarray | None = None, rec_every: int = 1, height: float = HEIGHT,
            distance: int = DISTANCE, precision: str = "fp32", chunk: int = 2000,
            score_dt: float | None = None):
    """The whole exploration on the GPU: the grid of ``gen_params``, one
    resident simulation of every grid point (``grid_simulation``) and the
    dV/dt peak count of each trace where it lies.  Returns (scores
    [len(p1_values), len(p2_values)] float64, the grid)."""
    grid = gen_params(base, p1, p1_values, p2, p2_values)
    sim, score_dt = grid_simulation(model, mapping, grid, stim, rec_every, precision, chunk, score_dt)
    counts = sim.dvdt_peaks(score_dt, 0, height, distance)
    n1 = grid.shape[0] // (len(p2_values) if p2_values is not None else NBINS)
    return counts.cpu().numpy().astype(np.float64).reshape(n1, -1), grid
